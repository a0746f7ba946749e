"""tn_heff_matvec_static (static device scratch, no allocation) against the
allocating tn_heff_matvec in FP64.  The entry point exists for callers that
cannot call cudaMalloc (their device memory is held by another allocator's
fixed pool, or their solver loop cannot take cudaMalloc's device-wide
synchronisation).  Collected last on purpose: it must pass both alone and
after every other test has used the library.

Tolerance: 1e-13 normwise relative (the same FP64 kernel chain runs in both;
the only difference is where its scratch lives)."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-13


@pytest.fixture(scope="module")
def T():
    import tensornetworks_b200 as T
    return T


@pytest.fixture(scope="module")
def ctx(T):
    return T.default_context()


def dev(x):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x, dtype=np.float64)).cuda()


@pytest.mark.parametrize("d,D1,D2,Dw1,Dw2", [(2, 64, 64, 5, 5), (2, 128, 96, 5, 5), (3, 48, 32, 5, 5),
                                              (2, 224, 224, 5, 5), (2, 1, 2, 1, 5), (2, 32, 16, 5, 1)])
def test_static_matvec_matches_allocating(T, ctx, oracle, d, D1, D2, Dw1, Dw2):
    import torch
    rng = np.random.default_rng(1000 * D1 + D2)
    W = oracle.mpo_site(10, (d - 1) / 2, 2, 1.0, 1.0, 0.3, 5 if (Dw1, Dw2) == (5, 5) else (1 if Dw1 == 1 else 10))
    assert W.shape[:2] == (Dw1, Dw2)
    Wc = np.ascontiguousarray(W.ravel())
    F, G = dev(rng.uniform(-1, 1, Dw1 * D1 * D1)), dev(rng.uniform(-1, 1, Dw2 * D2 * D2))
    lib = ctx._lib
    for call in range(2):  # two calls in a row, different vectors
        x = dev(rng.uniform(-1, 1, d * D1 * D2))
        y_ref = torch.zeros_like(x)
        y = torch.full_like(x, float("nan"))
        T._capi.check(lib.tn_heff_matvec(ctx.handle, 0, d, Dw1, Dw2, D1, D2, Wc.ctypes.data, F.data_ptr(),
                                         G.data_ptr(), x.data_ptr(), y_ref.data_ptr()), "tn_heff_matvec")
        T._capi.check(lib.tn_heff_matvec_static(ctx.handle, d, Dw1, Dw2, D1, D2, Wc.ctypes.data, F.data_ptr(),
                                                G.data_ptr(), x.data_ptr(), y.data_ptr()), "tn_heff_matvec_static")
        ctx.synchronize()
        a, b = y.cpu().numpy(), y_ref.cpu().numpy()
        assert np.all(np.isfinite(a))
        assert np.linalg.norm(a - b) <= TOL * np.linalg.norm(b), (call, np.linalg.norm(a - b) / np.linalg.norm(b))
        # and against the CPU oracle
        ref = oracle.heff_matvec(W, F.cpu().numpy(), G.cpu().numpy(), x.cpu().numpy(), D1, D2)
        assert np.linalg.norm(a - ref) <= 1e-12 * np.linalg.norm(ref)


def test_static_matvec_rejects_oversize(T, ctx, oracle):
    """D = 256 needs more than the static scratch: rejected before any launch."""
    W = np.ascontiguousarray(oracle.mpo_site(10, 0.5, 2, 1.0, 1.0, 0.0, 5).ravel())
    one = C.c_double(0.0)
    p = C.addressof(one)  # never dereferenced on this path
    st = ctx._lib.tn_heff_matvec_static(ctx.handle, 2, 5, 5, 256, 256, W.ctypes.data, p, p, p, p)
    assert st == 2  # TN_BAD_SHAPE
    assert "static" in T._capi.last_error()


def test_static_matvec_allocates_nothing(T, oracle):
    """Through a context of its own (no context buffers to fall back on), two
    calls in a row leave the device's free memory exactly as it was, and both
    agree with the allocating entry point run afterwards on the default
    context."""
    import torch
    d, D1, D2, Dw = 2, 160, 160, 5
    rng = np.random.default_rng(77)
    W = np.ascontiguousarray(oracle.mpo_site(10, 0.5, 2, 1.0, 1.0, 0.1, 5).ravel())
    F, G = dev(rng.uniform(-1, 1, Dw * D1 * D1)), dev(rng.uniform(-1, 1, Dw * D2 * D2))
    xs = [dev(rng.uniform(-1, 1, d * D1 * D2)) for _ in range(2)]
    ys = [torch.full_like(xs[0], float("nan")) for _ in range(2)]
    own = T.Context(0)
    try:
        lib = own._lib
        # warm-up on another array pair: the first call on a device looks up the array's address
        w = torch.zeros_like(xs[0])
        T._capi.check(lib.tn_heff_matvec_static(own.handle, d, Dw, Dw, D1, D2, W.ctypes.data, F.data_ptr(),
                                                G.data_ptr(), xs[0].data_ptr(), w.data_ptr()), "warm-up")
        own.synchronize()
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        for x, y in zip(xs, ys):
            T._capi.check(lib.tn_heff_matvec_static(own.handle, d, Dw, Dw, D1, D2, W.ctypes.data, F.data_ptr(),
                                                    G.data_ptr(), x.data_ptr(), y.data_ptr()),
                          "tn_heff_matvec_static")
            own.synchronize()
        free1 = torch.cuda.mem_get_info()[0]
        assert free1 == free0, (free0, free1)
    finally:
        own.close()
    ctx = T.default_context()
    for x, y in zip(xs, ys):
        y_ref = torch.zeros_like(x)
        T._capi.check(ctx._lib.tn_heff_matvec(ctx.handle, 0, d, Dw, Dw, D1, D2, W.ctypes.data, F.data_ptr(),
                                              G.data_ptr(), x.data_ptr(), y_ref.data_ptr()), "tn_heff_matvec")
        ctx.synchronize()
        a, b = y.cpu().numpy(), y_ref.cpu().numpy()
        assert np.linalg.norm(a - b) <= TOL * np.linalg.norm(b)
