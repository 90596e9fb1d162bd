"""GEMM tile forms pinned per process with NGW_TILES.

Split-K of GEMM1 summed inside a thread-block cluster (variants 5 and 6)
gives bit-identical Sigma_c to the same tiles with the separate reduction
kernel (variants 3 and 4): the same partial tiles summed in the same order.
Every GEMM2 form with the Clenshaw epilogue stays within 1 meV of the oracle."""
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r"""
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
np.save({out!r}, sig)
"""


def _run(tmp_path, tiles, **extra_env):
    out = str(tmp_path / ("sig_" + tiles.replace(",", "_") + "_".join(extra_env) + ".npy"))
    env = dict(os.environ, NGW_TILES=tiles, NGW_DENSE="0", **extra_env)   # the factored p(C) these tiles run
    subprocess.run([sys.executable, "-c", SCRIPT.format(root=ROOT, out=out)], env=env, check=True,
                   timeout=600)
    return np.load(out)


@pytest.mark.parametrize("plain,cluster", [("64,3,2,64,0", "64,5,2,64,0"), ("32,4,4,64,0", "32,6,4,64,0")])
def test_cluster_split_k_bit_identical(tmp_path, plain, cluster):
    a = _run(tmp_path, plain)
    b = _run(tmp_path, cluster)
    assert np.array_equal(a, b)


QP_SCRIPT = r"""
import sys, numpy as np
sys.path.insert(0, {root!r})
import nanogw_b200 as ngw
from tests._system import make_small_system
from oracle import sigma as OS
S = make_small_system()
qp = np.array([S.nval - 1, S.nval, S.nval + 1, S.nval + 2], dtype=np.int32)
nen, deltae, ecuts, niter = 81, 2.0, 0.02, 24
with ngw.Session(0, "mixed") as s:
    s.set_isdf(S.psi_intp, S.M)
    s.set_pairs(S.cvpair, S.sqrtR)
    got = s.calculate_sigma_lanczos(S.e1, S.nval, qp, nen, deltae, ecuts, niter, S.poly)
    sh = s.mixed_gemm_shapes(len(qp) * S.nmem)
refs = np.stack([OS.sigma_c_state(S.psi_intp, S.M, S.e1, S.nval, int(m), nen, deltae, ecuts, niter, S.poly)
                 for m in qp], axis=1)
sx, vx = np.full(len(qp), -0.4), np.full(len(qp), -0.6)
er = OS.qp_energies(refs.T, S.e1, S.e1, qp, deltae, sx, vx, xacc_ev=1e-7)
eg = OS.qp_energies(got.T, S.e1, S.e1, qp, deltae, sx, vx, xacc_ev=1e-7)
np.save({out!r}, np.array([abs(a[0] - b[0]) * 1e3 for a, b in zip(eg, er)] + [sh[10], sh[11]]))
"""


def _qp(tmp_path, tiles):
    out = str(tmp_path / ("qp_" + tiles.replace(",", "_") + ".npy"))
    env = dict(os.environ, NGW_TILES=tiles, NGW_DENSE="0")
    subprocess.run([sys.executable, "-c", QP_SCRIPT.format(root=ROOT, out=out)], env=env, check=True,
                   timeout=600)
    return np.load(out)


def test_cluster_split_k_gemm2_within_1mev(tmp_path):
    """GEMM2 with its K split across a 2-CTA cluster (Clenshaw epilogue on
    the cluster-summed tile): QP energies within 1 meV of the FP64 oracle."""
    r = _qp(tmp_path, "64,3,2,64,6,2")
    assert r[-2] == 6 and r[-1] == 2          # the pinned GEMM2 variant and split ran
    assert np.all(r[:-2] < 1.0), r


@pytest.mark.parametrize("gemm2", ["64,2", "64,3", "64,4", "32,4", "128,3", "32,6,4", "32,7", "64,7", "80,7", "256,1"])
def test_gemm2_variants_within_1mev(tmp_path, gemm2):
    """Every GEMM2 kernel form with the Clenshaw epilogue (persistent, fused
    one or two CTAs per SM, cluster split-K) keeps the QP energies within
    1 meV of the FP64 oracle."""
    r = _qp(tmp_path, "64,3,2," + gemm2)
    parts = [int(x) for x in gemm2.split(",")]
    assert r[-2] == parts[1] and r[-1] == (parts[2] if len(parts) > 2 else 1)
    assert np.all(r[:-2] < 1.0), r


def test_gemm2_occupancy_forms_bit_identical(tmp_path):
    """The fused GEMM2 at one and at two CTAs per SM, and with its Clenshaw
    operands staged by TMA (variant 7), runs the same MMAs and the same
    epilogue arithmetic: identical Sigma_c."""
    a = _run(tmp_path, "64,3,2,64,3")
    b = _run(tmp_path, "64,3,2,64,4")
    c = _run(tmp_path, "64,3,2,64,7")
    assert np.array_equal(a, b)
    assert np.array_equal(a, c)


@pytest.mark.parametrize("tiles", ["64,3,2,64,4", "64,3,2,96,1"])
def test_operand_ring_bit_identical(tmp_path, tiles):
    """GEMM2's Clenshaw operands through the TMA chunk ring or loaded by each
    thread (NGW_RING=0): the same values in the same arithmetic."""
    a = _run(tmp_path, tiles)
    b = _run(tmp_path, tiles, NGW_RING="0")
    assert np.array_equal(a, b)
