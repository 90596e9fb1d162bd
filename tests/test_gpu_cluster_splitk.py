"""Split-K of GEMM1 summed inside a thread-block cluster (variants 5 and 6)
gives bit-identical Sigma_c to the same tiles with the separate reduction
kernel (variants 3 and 4): the same partial tiles summed in the same order.
Tiles are pinned per process with NGW_TILES."""
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


def _run(tmp_path, tiles):
    out = str(tmp_path / ("sig_" + tiles.replace(",", "_") + ".npy"))
    env = dict(os.environ, NGW_TILES=tiles)
    subprocess.run([sys.executable, "-c", SCRIPT.format(root=ROOT, out=out)], env=env, check=True,
                   timeout=600)
    return np.load(out)


@pytest.mark.parametrize("plain,cluster", [("64,3,2,64,0", "64,5,2,64,0"), ("32,4,4,64,0", "32,6,4,64,0")])
def test_cluster_split_k_bit_identical(tmp_path, plain, cluster):
    a = _run(tmp_path, plain)
    b = _run(tmp_path, cluster)
    assert np.array_equal(a, b)
