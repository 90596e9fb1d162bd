"""A new chain count (or N_cv) close to an already tuned shape reuses that
shape's GEMM tiles instead of running the autotuner again (a request stream
brings new shapes with almost every molecule); NGW_TUNE_EXACT=1 tunes every
new shape.  The reused tiles give the same Sigma_c up to the summation-order
rounding of other tiles."""
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
qa = np.arange(1, 9, dtype=np.int32)          # 8 QP states: 8 x 32 chains
qb = np.arange(1, 10, dtype=np.int32)         # 9 QP states: 9 x 32 chains (12.5 % more)
with ngw.Session(0, "mixed") as s:
    s.set_isdf(S.psi_intp, S.M)
    s.set_pairs(S.cvpair, S.sqrtR)
    s.calculate_sigma_lanczos(S.e1, S.nval, qa, 41, 3.0, 0.02, 12, S.poly)
    sys.stderr.write("=== second shape ===\n"); sys.stderr.flush()
    sig = s.calculate_sigma_lanczos(S.e1, S.nval, qb, 41, 3.0, 0.02, 12, S.poly)
np.save({out!r}, sig)
"""


def _run(tmp_path, name, **extra):
    out = str(tmp_path / (name + ".npy"))
    env = dict(os.environ, NGW_TUNE_VERBOSE="1", **extra)
    env.pop("NGW_TILES", None)
    r = subprocess.run([sys.executable, "-c", SCRIPT.format(root=ROOT, out=out)], env=env, check=True,
                       timeout=600, capture_output=True, text=True)
    after = r.stderr.split("=== second shape ===", 1)[1]
    return np.load(out), after.count("tune gemm")


def test_nearby_shape_reuses_tiles(tmp_path):
    sig_reuse, tuned_reuse = _run(tmp_path, "reuse")
    sig_exact, tuned_exact = _run(tmp_path, "exact", NGW_TUNE_EXACT="1")
    assert tuned_reuse == 0
    assert tuned_exact > 0
    assert np.max(np.abs(sig_reuse - sig_exact)) <= 1e-4 * np.max(np.abs(sig_exact))
