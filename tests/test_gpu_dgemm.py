"""The FP64 tensor-core GEMM (``ngw_dgemm``, mma.sync m8n8k4 .f64) through the
C ABI against numpy's FP64 matmul on the same seeded inputs: every
transpose combination, ragged sizes, padded leading dimensions, both tile
sizes, split K with a workspace (slices summed in a fixed order: two calls
bit-identical), alpha / beta.  Bar: 1e-13 of |A| |B| per element.  The
throughput at a large square shape is printed beside torch's (cuBLAS)."""
import ctypes

import numpy as np
import pytest
import torch

from nanogw_b200._lib import check, lib

pytestmark = pytest.mark.gpu


def _dev(a):
    """a flat device buffer holding a in column-major order"""
    return torch.from_numpy(np.ascontiguousarray(np.asarray(a).ravel(order="F"))).cuda()


def _run(ta, tb, m, n, k, lda_pad=0, ldb_pad=0, ldc_pad=0, alpha=1.0, beta=0.0, ws=False, seed=0):
    rng = np.random.default_rng(seed)
    ar, ac = (k, m) if ta else (m, k)
    br, bc = (n, k) if tb else (k, n)
    A = np.zeros((ar + lda_pad, ac))
    B = np.zeros((br + ldb_pad, bc))
    C = np.zeros((m + ldc_pad, n))
    A[:ar] = rng.standard_normal((ar, ac))
    B[:br] = rng.standard_normal((br, bc))
    C[:m] = rng.standard_normal((m, n))
    dA, dB, dC = _dev(A), _dev(B), _dev(C)
    wsb = 64 * m * n * 8 if ws else 0
    dW = torch.empty(max(wsb // 8, 1), dtype=torch.float64, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    check(lib().ngw_dgemm(int(ta), int(tb), m, n, k, alpha, dA.data_ptr(), ar + lda_pad, dB.data_ptr(),
                          br + ldb_pad, beta, dC.data_ptr(), m + ldc_pad, dW.data_ptr() if ws else None,
                          wsb, ctypes.c_void_p(st)))
    torch.cuda.synchronize()
    got = dC.cpu().numpy().reshape(C.shape, order="F")
    opA = A[:ar].T if ta else A[:ar]
    opB = B[:br].T if tb else B[:br]
    ref = alpha * opA @ opB + beta * C[:m]
    scale = np.abs(opA) @ np.abs(opB)
    err = np.max(np.abs(got[:m] - ref) / (scale + 1.0))
    assert np.array_equal(got[m:], C[m:]), "rows past m of C were written"
    return err, got


@pytest.mark.parametrize("ta", [False, True])
@pytest.mark.parametrize("tb", [False, True])
def test_dgemm_transposes_ragged(ta, tb):
    err, _ = _run(ta, tb, 97, 61, 131, lda_pad=3, ldb_pad=5, ldc_pad=2, alpha=0.75, beta=-0.5)
    assert err < 1e-13, err


@pytest.mark.parametrize("ta,tb", [(False, False), (True, False), (False, True)])
def test_dgemm_large_tiles(ta, tb):
    err, _ = _run(ta, tb, 1100, 900, 300, seed=1)      # 128 x 128 tile path
    assert err < 1e-13, err


def test_dgemm_split_k_deterministic():
    e1, g1 = _run(True, False, 40, 24, 9000, ws=True, seed=2)
    e2, g2 = _run(True, False, 40, 24, 9000, ws=True, seed=2)
    e3, _ = _run(True, False, 40, 24, 9000, ws=False, seed=2)
    assert e1 < 1e-13 and e3 < 1e-13
    assert np.array_equal(g1, g2)


def test_dgemm_throughput_large_square():
    n = 4096
    A = torch.randn(n, n, dtype=torch.float64, device="cuda")
    B = torch.randn(n, n, dtype=torch.float64, device="cuda")
    C = torch.empty(n, n, dtype=torch.float64, device="cuda")
    st = torch.cuda.current_stream().cuda_stream

    def ours():
        check(lib().ngw_dgemm(0, 0, n, n, n, 1.0, A.data_ptr(), n, B.data_ptr(), n, 0.0, C.data_ptr(), n,
                              None, 0, ctypes.c_void_p(st)))

    def theirs():
        torch.matmul(A, B, out=C)

    out = {}
    for name, f in (("ngw_dgemm", ours), ("torch/cuBLAS", theirs)):
        for _ in range(2):
            f()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(5):
            f()
        e1.record()
        torch.cuda.synchronize()
        out[name] = 2.0 * n ** 3 * 5 / (e0.elapsed_time(e1) * 1e-3) / 1e12
    print("FP64 GEMM 4096^3 TFLOP/s:", out)
    assert out["ngw_dgemm"] > 5.0
