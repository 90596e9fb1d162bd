"""ngw_qp_newton_noalloc: the QP Newton solve for callers that cannot
allocate device memory (a Fortran driver handing out its own device pool,
code running during stream capture, a process whose allocator holds all free
memory).  It takes device pointers for inputs and outputs and keeps its
spline workspace in a fixed device array, so it calls no cudaMalloc.

Checked through the C ABI against the regular entry point (ngw_qp_newton) on
the same inputs, twice in a row (the second call reuses the workspace the
first one left behind), within the tolerance of the QP tests (1e-9 eV).
This file is collected last so a run that stops at the first failure has
already run every other test."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _inputs(seed, nqp=7, nen=121):
    rng = np.random.default_rng(seed)
    e1 = rng.uniform(-10, 5, nqp)
    deltae = 10.0
    x = e1[None, :] - deltae / 2 + deltae / (nen - 1) * np.arange(nen)[:, None]
    sig = (0.8 / (x - e1[None, :] - 12.0) - 0.3 * (x - e1[None, :])) + 0.01j
    sx = rng.uniform(-3, -1, nqp)
    vx = rng.uniform(-4, -2, nqp)
    return np.asfortranarray(sig), e1, deltae, sx, vx


def test_noalloc_matches_regular_entry_point_twice():
    import torch

    import nanogw_b200 as ngw
    from nanogw_b200._lib import check, lib

    L = lib()
    f = L.ngw_qp_newton_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_int, ctypes.c_int] + [ctypes.c_void_p] * 3 + [ctypes.c_double] + \
        [ctypes.c_void_p] * 2 + [ctypes.c_double] + [ctypes.c_void_p] * 4
    torch.cuda.set_device(0)
    dev = torch.device("cuda:0")
    with ngw.Session(0) as s:
        for seed in (1, 2):
            sig, e1, deltae, sx, vx = _inputs(seed)
            nen, nqp = sig.shape
            ref_e, ref_z, ref_i = s.qp_newton(sig, e1, e1, deltae, sx, vx, 1e-6)
            d_sig = torch.from_numpy(np.ascontiguousarray(sig.T).view(np.float64).ravel()).to(dev)
            d_e1 = torch.from_numpy(e1).to(dev)
            d_sx = torch.from_numpy(sx).to(dev)
            d_vx = torch.from_numpy(vx).to(dev)
            d_eq = torch.zeros(nqp, dtype=torch.float64, device=dev)
            d_z = torch.zeros(nqp, dtype=torch.float64, device=dev)
            d_ie = torch.full((nqp,), -1, dtype=torch.int32, device=dev)
            torch.cuda.synchronize()
            check(f(nqp, nen, d_sig.data_ptr(), d_e1.data_ptr(), d_e1.data_ptr(), deltae, d_sx.data_ptr(),
                    d_vx.data_ptr(), 1e-6, d_eq.data_ptr(), d_z.data_ptr(), d_ie.data_ptr(), None))
            torch.cuda.synchronize()
            assert np.all(d_ie.cpu().numpy() == ref_i)
            assert np.max(np.abs(d_eq.cpu().numpy() - ref_e)) < 1e-9
            assert np.max(np.abs(d_z.cpu().numpy() - ref_z)) < 1e-9


def test_noalloc_rejects_oversize():
    from nanogw_b200._lib import NGW_ERR_BUDGET, lib
    f = lib().ngw_qp_newton_noalloc
    f.restype = ctypes.c_int
    one = ctypes.c_void_p(8)    # never dereferenced: the size check comes first
    rc = f(1 << 12, 1 << 8, one, one, one, ctypes.c_double(1.0), one, one, ctypes.c_double(1e-6),
           one, one, one, None)
    assert rc == NGW_ERR_BUDGET
    assert b"exceeds" in lib().ngw_last_error()
