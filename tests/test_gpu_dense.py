"""Dense p(C) form of the mixed path (small N_cv): H = P_perp p(Chat_perp)
formed once in FP64 and applied as one split-BF16 tcgen05 GEMM per Lanczos
step, the deflated eigenpairs added in FP64 in the epilogue.  It computes the
same p(C) v as the factored Clenshaw form (NGW_DENSE=0), so on the stable
(reorthogonalised) recurrence both agree with each other and with the FP64
oracle to the split-BF16 rounding."""
import os

import numpy as np
import pytest

import nanogw_b200 as ngw
from oracle import lanczos as L
from oracle import sigma as OS

pytestmark = pytest.mark.gpu


@pytest.fixture()
def env():
    saved = dict(os.environ)
    yield os.environ
    os.environ.clear()
    os.environ.update(saved)


def _session(S, precision="mixed"):
    s = ngw.Session(0, precision)
    s.set_isdf(S.psi_intp, S.M)
    s.set_pairs(S.cvpair, S.sqrtR)
    return s


def _rel(a, b):
    return np.max(np.abs(a - b)) / np.max(np.abs(b))


def test_dense_first_product_vs_oracle(small_system, env):
    """alpha_1 = <v|p(C)|v> of every chain: dense mixed form against the FP64
    oracle's polynomial, to the split-BF16 rounding."""
    S = small_system
    env["NGW_DENSE"] = "1"
    p, pn2 = OS.start_vectors(S.psi_intp, S.M, S.Cmtrx, S.sqrtR, S.nval, np.arange(1, 9))
    zz = np.repeat((np.linspace(-1.0, 1.0, 5) + 0.02j)[:, None], 8, 1)
    _, a_r, b_r = L.lanczos_spectra_isdf(p, np.sqrt(pn2), zz, 2, S.poly, S.Cmtrx, S.M, S.sqrtR)
    with _session(S) as s:
        _, a, b = s.lanczos_spectra_isdf(p, np.sqrt(pn2), zz, 2, S.poly)
        assert s.profile_dense_gemm(8, reps=2) is not None
    assert np.max(np.abs(a[0] - a_r[0]) / np.abs(a_r[0])) < 1e-4


def test_dense_equals_factored_and_oracle(small_system, env):
    """Sigma_c with full reorthogonalisation: dense and factored mixed forms
    against each other and the FP64 oracle; QP energies within 0.1 meV."""
    S = small_system
    qp = np.array([S.nval - 1, S.nval, S.nval + 1, S.nval + 2], dtype=np.int32)
    nen, deltae, ecuts, niter = 41, 2.0, 0.02, 20
    out = {}
    for mode in ("0", "1"):
        env["NGW_DENSE"] = mode
        with _session(S) as s:
            out[mode] = s.calculate_sigma_lanczos(S.e1, S.nval, qp, nen, deltae, ecuts, niter, S.poly,
                                                  reorth=True)
            if mode == "0":
                assert s.profile_dense_gemm(len(qp) * S.nmem, reps=2) is None
    refs = np.stack([OS.sigma_c_state(S.psi_intp, S.M, S.e1, S.nval, int(m), nen, deltae, ecuts, niter,
                                      S.poly, reorth=True) for m in qp], axis=1)
    print("dense vs factored", _rel(out["1"], out["0"]), "dense vs oracle", _rel(out["1"], refs),
          "factored vs oracle", _rel(out["0"], refs))
    assert _rel(out["1"], refs) < 1e-3
    sigx = np.full(len(qp), -0.4)
    vxc = np.full(len(qp), -0.6)
    e = {k: OS.qp_energies(v.T, S.e1, S.e1, qp, deltae, sigx, vxc, xacc_ev=1e-7) for k, v in out.items()}
    e_ref = OS.qp_energies(refs.T, S.e1, S.e1, qp, deltae, sigx, vxc, xacc_ev=1e-7)
    for k in e:
        err = np.array([abs(a[0] - b[0]) * 1e3 for a, b in zip(e[k], e_ref)])
        print("NGW_DENSE", k, "QP error vs oracle (meV)", err)
        assert np.all(err < 0.1)


def test_dense_plain_recurrence_qp(small_system, env):
    """The reference (unreorthogonalised) recurrence through the dense form:
    QP energies against the FP64 oracle within 1 meV."""
    S = small_system
    env["NGW_DENSE"] = "1"
    qp = np.array([S.nval - 1, S.nval, S.nval + 1, S.nval + 2], dtype=np.int32)
    nen, deltae, ecuts, niter = 81, 2.0, 0.02, 24
    with _session(S) as s:
        got = s.calculate_sigma_lanczos(S.e1, S.nval, qp, nen, deltae, ecuts, niter, S.poly)
    refs = np.stack([OS.sigma_c_state(S.psi_intp, S.M, S.e1, S.nval, int(m), nen, deltae, ecuts, niter,
                                      S.poly) for m in qp], axis=1)
    sigx = np.full(len(qp), -0.4)
    vxc = np.full(len(qp), -0.6)
    e_ref = OS.qp_energies(refs.T, S.e1, S.e1, qp, deltae, sigx, vxc, xacc_ev=1e-7)
    e_got = OS.qp_energies(got.T, S.e1, S.e1, qp, deltae, sigx, vxc, xacc_ev=1e-7)
    err = np.array([abs(a[0] - b[0]) * 1e3 for a, b in zip(e_got, e_ref)])
    print("dense plain recurrence QP error (meV):", err)
    assert np.all(err < 1.0)


DENSE_SCRIPT = r"""
import sys, numpy as np
sys.path.insert(0, {root!r})
import nanogw_b200 as ngw
from tests._system import make_small_system
S = make_small_system()
with ngw.Session(0, "mixed") as s:
    s.set_isdf(S.psi_intp, S.M)
    s.set_pairs(S.cvpair, S.sqrtR)
    qp = np.array([S.nval - 1, S.nval, S.nval + 1, S.nval + 2], dtype=np.int32)
    sig = s.calculate_sigma_lanczos(S.e1, S.nval, qp, 41, 3.0, 0.02, 20, S.poly)
    shape = s.profile_dense_gemm(len(qp) * S.nmem, reps=2)[1]
np.save({out!r}, np.concatenate([sig.ravel().view(np.float64), np.array(shape, dtype=np.float64)]))
"""


def test_dense_occupancy_forms_bit_identical(tmp_path):
    """The dense GEMM fused at one and at two CTAs per SM (NGW_DENSE_TILES
    64,3 and 64,4) runs the same MMAs and epilogue: identical Sigma_c."""
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = {}
    for tiles in ("64,3", "64,4"):
        f = str(tmp_path / ("dense_" + tiles.replace(",", "_") + ".npy"))
        env = dict(os.environ, NGW_DENSE="1", NGW_DENSE_TILES=tiles)
        subprocess.run([sys.executable, "-c", DENSE_SCRIPT.format(root=root, out=f)], env=env, check=True,
                       timeout=600)
        out[tiles] = np.load(f)
    assert out["64,3"][-2] == 64 and out["64,4"][-2] == 64
    assert out["64,3"][-1] == 3 * 16 + 1 and out["64,4"][-1] == 4 * 16 + 1
    assert np.array_equal(out["64,3"][:-5], out["64,4"][:-5])
