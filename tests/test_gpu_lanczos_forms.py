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
    env = dict(os.environ, NGW_TILES="64,3,2,64,4", NGW_DENSE="0", **env_extra)   # same GEMM tiles in both runs
    subprocess.run([sys.executable, "-c", SCRIPT.format(root=ROOT, out=out)], env=env, check=True,
                   timeout=600)
    return np.load(out)


def test_register_and_three_pass_step_identical(tmp_path):
    a = _run(tmp_path, "reg", NGW_LSTEP="r")
    b = _run(tmp_path, "pass3", NGW_LSTEP="3")
    assert np.array_equal(a, b)


SCRIPT_RANDOM = r"""
import sys, numpy as np
sys.path.insert(0, {root!r})
import nanogw_b200 as ngw
from nanogw_b200.api import lowcomsym_pairs, sqrt_r
from nanogw_b200.polyfit import sigma_polynomial
nocc, nemp, n_isdf = {nocc}, {nemp}, {n_isdf}
rng = np.random.default_rng(5)
nmem = nocc + nemp
psi = np.asfortranarray(rng.standard_normal((n_isdf, nmem)) * 0.05)
g = rng.standard_normal((n_isdf, n_isdf)) / np.sqrt(n_isdf)
M = np.asfortranarray(g @ g.T * 0.02)
e1 = np.sort(np.concatenate([rng.uniform(-1.5, -0.5, nocc), rng.uniform(-0.3, 1.0, nemp)]))
cv = lowcomsym_pairs(nocc, nmem)
poly = sigma_polynomial(e1, nocc, nmem, 12)[0]
qp = np.array([nocc, nocc + 1], dtype=np.int32)
out = []
for prec in ("fp64", "mixed"):
    with ngw.Session(0, prec) as s:
        s.set_isdf(psi, M)
        s.set_pairs(cv, sqrt_r(e1, cv))
        sig, a, b = s.calculate_sigma_lanczos(e1, nocc, qp, 41, 3.0, 0.02, 12, poly, return_ab=True)
    out += [sig.real.ravel(), sig.imag.ravel(), a.ravel(), b.ravel()]
np.save({out!r}, np.concatenate(out))
"""


@pytest.mark.parametrize("nocc,nemp", [(25, 200), (28, 250)])
def test_register_forms_of_production_sizes(tmp_path, nocc, nemp):
    """The register step's 24- and 32-element instantiations, which the
    default picks for 4096 < N_cv <= 6144 and 6144 < N_cv <= 8192 (here
    N_cv = 5000 and 7000 on random operators), against the three-pass form:
    identical alpha, beta and Sigma_c in both precisions."""
    res = []
    for mode in ("r", "3"):
        out = str(tmp_path / f"{mode}.npy")
        env = dict(os.environ, NGW_TILES="64,3,2,64,4", NGW_DENSE="0", NGW_LSTEP=mode)
        code = SCRIPT_RANDOM.format(root=ROOT, out=out, nocc=nocc, nemp=nemp, n_isdf=200)
        subprocess.run([sys.executable, "-c", code], env=env, check=True, timeout=600)
        res.append(np.load(out))
    assert np.array_equal(res[0], res[1])
