"""A new chain count (or N_cv) close to an already tuned shape reuses that
shape's GEMM tiles instead of running the autotuner again (a request stream
brings new shapes with almost every molecule); NGW_TUNE_EXACT=1 tunes every
new shape.  Other tiles sum in another order; through the unreorthogonalised
recurrence that moves Sigma_c(omega) near its poles, so the comparison is on
the QP energies, which agree within 1 meV."""
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
from oracle import sigma as OS
S = make_small_system()
qa = np.arange(S.nval - 3, S.nval + 5, dtype=np.int32)   # 8 QP states near the gap: 8 x 32 chains
qb = np.arange(S.nval - 3, S.nval + 6, dtype=np.int32)   # 9 states: 12.5 % more chains
with ngw.Session(0, "mixed") as s:
    s.set_isdf(S.psi_intp, S.M)
    s.set_pairs(S.cvpair, S.sqrtR)
    s.calculate_sigma_lanczos(S.e1, S.nval, qa, 81, 2.0, 0.02, 24, S.poly)
    sys.stderr.write("=== second shape ===\n"); sys.stderr.flush()
    sig = s.calculate_sigma_lanczos(S.e1, S.nval, qb, 81, 2.0, 0.02, 24, S.poly)
sx, vx = np.full(len(qb), -0.4), np.full(len(qb), -0.6)
eq = OS.qp_energies(sig.T, S.e1, S.e1, qb, 2.0, sx, vx, xacc_ev=1e-7)
np.save({out!r}, np.array([e[0] for e in eq]))
"""


def _run(tmp_path, name, **extra):
    out = str(tmp_path / (name + ".npy"))
    env = dict(os.environ, NGW_TUNE_VERBOSE="1", NGW_DENSE="0", **extra)   # the factored GEMMs' tuner
    env.pop("NGW_TILES", None)
    r = subprocess.run([sys.executable, "-c", SCRIPT.format(root=ROOT, out=out)], env=env, check=True,
                       timeout=600, capture_output=True, text=True)
    after = r.stderr.split("=== second shape ===", 1)[1]
    return np.load(out), after.count("tune gemm")


def test_nearby_shape_reuses_tiles(tmp_path):
    e_reuse, tuned_reuse = _run(tmp_path, "reuse")
    e_exact, tuned_exact = _run(tmp_path, "exact", NGW_TUNE_EXACT="1")
    assert tuned_reuse == 0
    assert tuned_exact > 0
    assert np.all(np.abs(e_reuse - e_exact) * 1e3 < 1.0), (e_reuse, e_exact)   # eV -> meV
