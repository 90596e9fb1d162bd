"""Batched Sigma_c across molecules of uneven size (ngw_sigma_lanczos_batch).

* Branch mode (the default): one graph whose branches are the molecules'
  solves; each entry bit-identical to the same session's single call,
  through the eager first call, the capture and the replays (these small
  molecules take the dense p(C) form).
* Grouped mode (NGW_BATCH_MODE=grouped): the molecules' recurrences in lock
  step, each Clenshaw term one grouped GEMM1 and one grouped GEMM2 launch
  over all of them, one grouped Lanczos-step launch per step.  With the
  single calls pinned to the grouped tiles (64-wide, fused stages, no
  split-K) the results are bit-identical; with the single calls on their own
  tuned tiles they agree to the mixed form's rounding (QP energies within
  1 meV).
Per-chain lengths ride along (entry 1), so the grouped launches shrink as
that molecule's chains finish."""
import os

import numpy as np
import pytest

import nanogw_b200 as ngw
from nanogw_b200 import pipeline, synth
from nanogw_b200.polyfit import sigma_polynomial

pytestmark = pytest.mark.gpu


def _molecule(seed, n_atoms, R, nocc, nemp, n_isdf):
    mol = synth.make_molecule(n_atoms, 2.5, R, 0.5, nocc, nemp, seed)
    with ngw.Session(0) as s:
        op = pipeline.build_operator(mol, n_isdf, s, qp_bands=pipeline.qp_bands_near_gap(mol.nval, 4),
                                     seed=seed)
    poly, _, _ = sigma_polynomial(op.e1, op.nval, op.nmem, 12)
    return op, poly


@pytest.fixture(scope="module")
def molecules():
    return [_molecule(31, 4, 5.0, 8, 24, 96), _molecule(32, 6, 6.0, 12, 40, 128),
            _molecule(33, 5, 5.5, 10, 30, 110)]


@pytest.fixture()
def env():
    saved = dict(os.environ)
    yield os.environ
    os.environ.clear()
    os.environ.update(saved)


@pytest.mark.parametrize("precision,mode", [("fp64", "branches"), ("mixed", "branches"),
                                            ("mixed", "grouped_pinned")])
def test_batch_equals_single_calls(molecules, precision, mode, env):
    if mode == "grouped_pinned":
        env["NGW_BATCH_MODE"] = "grouped"
        env["NGW_DENSE"] = "0"                # grouped launches run the factored p(C)
        env["NGW_TILES"] = "64,3,1,64,3"      # the grouped launches' tiles for the single calls
    sessions = []
    reqs = []
    try:
        for i, (op, poly) in enumerate(molecules):
            s = ngw.Session(0, precision)
            s.set_isdf(op.psi_intp, op.mmtrx)
            cv, sr = op.pairs()
            s.set_pairs(cv, sr)
            qp = pipeline.qp_bands_near_gap(op.nval, 4)
            req = dict(e1=op.e1, nval=op.nval, qp_bands=qp, nen=31, deltae=3.0, ecuts=0.02,
                       niter=20, polynomial=poly)
            if i == 1:      # uneven per-chain lengths on one entry
                req["chain_niter"] = np.random.default_rng(4).integers(6, 21, (len(qp), op.nmem))
            sessions.append(s)
            reqs.append(req)
        single = [s.calculate_sigma_lanczos(**r) for s, r in zip(sessions, reqs)]
        for _ in range(3):                       # eager, captured, replayed
            got = ngw.sigma_lanczos_batch(sessions, reqs)
            for g, r in zip(got, single):
                np.testing.assert_array_equal(g, r)
    finally:
        for s in sessions:
            s.close()


def test_batch_rejects_repeated_session(molecules):
    op, poly = molecules[0]
    with ngw.Session(0) as s:
        s.set_isdf(op.psi_intp, op.mmtrx)
        cv, sr = op.pairs()
        s.set_pairs(cv, sr)
        req = dict(e1=op.e1, nval=op.nval, qp_bands=pipeline.qp_bands_near_gap(op.nval, 2), nen=11,
                   deltae=3.0, ecuts=0.02, niter=4, polynomial=poly)
        with pytest.raises(ngw.NGWError) as e:
            ngw.sigma_lanczos_batch([s, s], [req, req])
        assert e.value.code == ngw._lib.NGW_ERR_ARG


def test_grouped_batch_matches_tuned_single_calls(molecules, env):
    """Default grouped batch against single calls on their own tuned tiles:
    the same polynomial, deflation and FP64 recurrence, only the BF16 tile
    arithmetic differs -> QP energies within 1 meV."""
    RYD = 13.60569193
    env["NGW_BATCH_MODE"] = "grouped"
    env["NGW_DENSE"] = "0"
    sessions, reqs = [], []
    try:
        for op, poly in molecules:
            s = ngw.Session(0, "mixed")
            s.set_isdf(op.psi_intp, op.mmtrx)
            cv, sr = op.pairs()
            s.set_pairs(cv, sr)
            qp = pipeline.qp_bands_near_gap(op.nval, 4)
            reqs.append(dict(e1=op.e1, nval=op.nval, qp_bands=qp, nen=101, deltae=3.0, ecuts=0.02, niter=40,
                             polynomial=poly))
            sessions.append(s)
        single = [s.calculate_sigma_lanczos(**r) for s, r in zip(sessions, reqs)]
        for _ in range(3):
            got = ngw.sigma_lanczos_batch(sessions, reqs)
        for s, r, g, a in zip(sessions, reqs, got, single):
            e1 = r["e1"][r["qp_bands"] - 1] * RYD
            eg = s.qp_newton(g * RYD, e1, e1, r["deltae"] * RYD, -5.0, -4.0, 1e-7)[0]
            ea = s.qp_newton(a * RYD, e1, e1, r["deltae"] * RYD, -5.0, -4.0, 1e-7)[0]
            err = np.abs(eg - ea) * 1e3
            print("grouped vs single QP (meV):", err)
            assert np.all(err < 1.0)
    finally:
        for s in sessions:
            s.close()
