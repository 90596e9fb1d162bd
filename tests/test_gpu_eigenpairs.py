"""Top eigenpairs of the Casida operator (the pairs the mixed path deflates)
from the persistent FP64 Lanczos kernel, through the C ABI, against the
dense eigen-decomposition of the oracle's operator.

A full-length run (msteps = ncv) spans the whole space: every Ritz value is
an eigenvalue to 1e-10 relative.  A short run gives Ritz values within their
residual bounds of the top eigenvalues.  The kernel's partitions and
summation orders are fixed, so two runs agree bit for bit; the cuBLAS form
of the same loop (NGW_EIG_BLAS=1) agrees to 1e-10 on converged pairs."""
import os
import subprocess
import sys

import numpy as np
import pytest

import nanogw_b200 as ngw
from oracle import lanczos as L

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def sess(small_system):
    s = ngw.Session(0, "fp64")
    s.set_isdf(small_system.psi_intp, small_system.M)
    s.set_pairs(small_system.cvpair, small_system.sqrtR)
    yield s
    s.close()


def _dense(S, tda):
    ncv = len(S.sqrtR)
    H = L.matvec_isdf(np.eye(ncv), S.Cmtrx, S.M, S.sqrtR, tamm_d=tda)
    return np.sort(np.linalg.eigvalsh(0.5 * (H + H.T)))[::-1]


@pytest.mark.parametrize("tda", [False, True])
def test_full_run_gives_the_spectrum(sess, small_system, tda):
    S = small_system
    ncv = len(S.sqrtR)
    lam = _dense(S, tda)
    vals, res = sess.operator_eigenpairs(kmax=16, msteps=ncv, tamm_d=tda)
    assert len(vals) == 16
    assert np.all(np.diff(vals) <= 0)
    assert np.max(np.abs(vals - lam[:16])) < 1e-10 * lam[0]


def test_short_run_within_residual_bounds(sess, small_system):
    S = small_system
    lam = _dense(S, False)
    vals, res = sess.operator_eigenpairs(kmax=8, msteps=60)
    assert len(vals) == 8
    for i in range(4):
        assert abs(vals[i] - lam[i]) <= res[i] + 1e-10 * lam[0], (i, vals[i], lam[i], res[i])
        assert vals[i] <= lam[i] + 1e-10 * lam[0]          # Ritz values interlace from below


def test_deterministic(sess):
    a = sess.operator_eigenpairs(kmax=16, msteps=100)
    b = sess.operator_eigenpairs(kmax=16, msteps=100)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


SCRIPT = r"""
import sys, numpy as np
sys.path.insert(0, {root!r})
import nanogw_b200 as ngw
from tests._system import make_small_system
S = make_small_system()
with ngw.Session(0, "fp64") as s:
    s.set_isdf(S.psi_intp, S.M)
    s.set_pairs(S.cvpair, S.sqrtR)
    v, r = s.operator_eigenpairs(kmax=16, msteps=100)
np.save({out!r}, np.stack([v, r]))
"""


def test_blas_loop_agrees(tmp_path, sess):
    out = str(tmp_path / "eig_blas.npy")
    env = dict(os.environ, NGW_EIG_BLAS="1")
    subprocess.run([sys.executable, "-c", SCRIPT.format(root=ROOT, out=out)], env=env, check=True,
                   timeout=600)
    vb, rb = np.load(out)
    v, r = sess.operator_eigenpairs(kmax=16, msteps=100)
    conv = (r < 1e-8 * v[0]) & (rb < 1e-8 * v[0])
    assert conv[:4].all()
    assert np.max(np.abs(v[conv] - vb[conv])) < 1e-10 * v[0]


def test_mixed_plan_recomputes_after_query(small_system):
    """A query with other Lanczos settings leaves the mixed path's own
    eigenpairs (and so its Sigma_c) unchanged."""
    S = small_system
    qp = np.array([S.nval, S.nval + 1], dtype=np.int32)
    with ngw.Session(0, "mixed") as s:
        s.set_isdf(S.psi_intp, S.M)
        s.set_pairs(S.cvpair, S.sqrtR)
        a = s.calculate_sigma_lanczos(S.e1, S.nval, qp, 21, 2.0, 0.02, 12, S.poly)
        s.operator_eigenpairs(kmax=4, msteps=30)
        b = s.calculate_sigma_lanczos(S.e1, S.nval, qp, 21, 2.0, 0.02, 12, S.poly)
    assert np.array_equal(a, b)


def test_barrier_wait_runs_out_and_session_recovers(small_system):
    """The persistent eigen kernel's grid barrier with a short wait bound
    (NGW_WAIT_CYCLES, ~1 ms) and one CTA withholding its first arrival
    (NGW_TEST_EIG_SKIP_ARRIVAL): every CTA's wait runs out, the kernel
    returns, the call reports NGW_ERR_TIMEOUT, and the same session then
    computes the eigenpairs and a mixed-precision solve exactly as a fresh
    session does.  Nothing asynchronous is in flight in this kernel."""
    from nanogw_b200._lib import NGW_ERR_TIMEOUT
    S = small_system
    with ngw.Session(0, "mixed") as s:
        s.set_isdf(S.psi_intp, S.M)
        s.set_pairs(S.cvpair, S.sqrtR)
        os.environ["NGW_WAIT_CYCLES"] = str(1 << 21)
        os.environ["NGW_TEST_EIG_SKIP_ARRIVAL"] = "0"
        try:
            with pytest.raises(ngw.NGWError) as ei:
                s.operator_eigenpairs(kmax=8, msteps=64)
        finally:
            del os.environ["NGW_WAIT_CYCLES"]
            del os.environ["NGW_TEST_EIG_SKIP_ARRIVAL"]
        assert ei.value.code == NGW_ERR_TIMEOUT
        vals, res = s.operator_eigenpairs(kmax=8, msteps=64)
        qp = np.array([S.nval, S.nval + 1], dtype=np.int32)
        sig = s.calculate_sigma_lanczos(S.e1, S.nval, qp, 41, 2.0, 0.02, 12, S.poly)
    with ngw.Session(0, "mixed") as f:
        f.set_isdf(S.psi_intp, S.M)
        f.set_pairs(S.cvpair, S.sqrtR)
        vals_f, res_f = f.operator_eigenpairs(kmax=8, msteps=64)
        sig_f = f.calculate_sigma_lanczos(S.e1, S.nval, qp, 41, 2.0, 0.02, 12, S.poly)
    assert np.array_equal(vals, vals_f) and np.array_equal(res, res_f)
    assert np.array_equal(sig, sig_f)
