"""CUDA-graph replay of the Sigma_c region after the operator changes.

The per-block region is run eagerly, captured on its second call and
replayed afterwards.  An operator of the same shapes is uploaded into the
existing device buffers (captured graphs stay valid and read the new values);
one of other shapes reallocates and drops every graph.  Either way the result
after the swap equals a fresh session's result for the new operator."""
import numpy as np
import pytest

import nanogw_b200 as ngw

pytestmark = pytest.mark.gpu


def _upload(s, S, M):
    s.set_isdf(S.psi_intp, M)
    s.set_pairs(S.cvpair, S.sqrtR)


def _sigma(s, S, niter=16):
    qp = np.array([S.nval, S.nval + 1], dtype=np.int32)
    return s.calculate_sigma_lanczos(S.e1, S.nval, qp, 31, 3.0, 0.02, niter, S.poly)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_operator_swap_drops_graphs(small_system, precision):
    S = small_system
    M2 = np.asfortranarray(S.M * 1.07)
    with ngw.Session(0, precision) as fresh:
        _upload(fresh, S, M2)
        ref = _sigma(fresh, S)
    with ngw.Session(0, precision) as s:
        _upload(s, S, S.M)
        runs = [_sigma(s, S) for _ in range(3)]       # eager, captured, replayed
        pad = ngw.Session(0, precision)               # other allocations between the operators
        pad.set_isdf(S.psi_intp, S.M)
        _upload(s, S, M2)
        got = [_sigma(s, S) for _ in range(3)]
        _upload(s, S, S.M)                            # back to the first operator, in place
        back = _sigma(s, S)
        pad.close()
    a = runs[0]
    np.testing.assert_array_equal(runs[1], a)
    np.testing.assert_array_equal(runs[2], a)
    assert not np.array_equal(a, got[0])
    for g in got:
        np.testing.assert_array_equal(g, ref)
    np.testing.assert_array_equal(back, a)
