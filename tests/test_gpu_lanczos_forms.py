"""The Lanczos step with each chain's vectors held in registers (forced with
NGW_LSTEP=r; by default used for 4096 < N_cv <= 8192) and the three-pass form
(NGW_LSTEP=3) run the same arithmetic in the same order: identical alpha,
beta and Sigma_c, in the FP64 and in the mixed-precision path."""
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
qp = np.array([S.nval - 1, S.nval, S.nval + 1], dtype=np.int32)
out = []
for prec in ("fp64", "mixed"):
    with ngw.Session(0, prec) as s:
        s.set_isdf(S.psi_intp, S.M)
        s.set_pairs(S.cvpair, S.sqrtR)
        sig, a, b = s.calculate_sigma_lanczos(S.e1, S.nval, qp, 41, 3.0, 0.02, 16, S.poly, return_ab=True)
    out += [sig.real.ravel(), sig.imag.ravel(), a.ravel(), b.ravel()]
np.save({out!r}, np.concatenate(out))
"""


def _run(tmp_path, name, **env_extra):
    out = str(tmp_path / (name + ".npy"))
    env = dict(os.environ, NGW_TILES="64,3,2,64,4", **env_extra)   # same GEMM tiles in both runs
    subprocess.run([sys.executable, "-c", SCRIPT.format(root=ROOT, out=out)], env=env, check=True,
                   timeout=600)
    return np.load(out)


def test_register_and_three_pass_step_identical(tmp_path):
    a = _run(tmp_path, "reg", NGW_LSTEP="r")
    b = _run(tmp_path, "pass3", NGW_LSTEP="3")
    assert np.array_equal(a, b)
