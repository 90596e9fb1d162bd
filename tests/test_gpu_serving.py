"""Continuous batching on the device: each request's result is the same
alone and in a mix of concurrently running requests (different molecule
sizes, overlapping on separate streams)."""
import numpy as np
import pytest

import nanogw_b200 as ngw
from nanogw_b200 import pipeline, synth
from nanogw_b200.polyfit import sigma_polynomial
from nanogw_b200.serving import SigmaRequest, SigmaServer

pytestmark = pytest.mark.gpu


def _molecule_request(rid, seed, n_atoms, R, nocc, nemp, n_isdf, nqp=4, niter=40):
    mol = synth.make_molecule(n_atoms, 2.5, R, 0.5, nocc, nemp, seed)
    qp = pipeline.qp_bands_near_gap(mol.nval, nqp)
    with ngw.Session(0) as s:
        op = pipeline.build_operator(mol, n_isdf, s, qp_bands=qp, seed=seed)
    poly, _, _ = sigma_polynomial(op.e1, op.nval, op.nmem, 12)
    return SigmaRequest(rid=rid, mol_id=seed, psi_intp=op.psi_intp, mmtrx=op.mmtrx, e1=op.e1,
                        nval=op.nval, qp_bands=qp, polynomial=poly, niter=niter, nen=101, deltae=3.0)


@pytest.fixture(scope="module")
def requests():
    return [_molecule_request(0, 21, 4, 5.0, 8, 24, 96),
            _molecule_request(1, 22, 6, 6.0, 12, 36, 120),
            _molecule_request(2, 23, 5, 5.5, 10, 40, 110)]


def _clone(r):
    return SigmaRequest(rid=r.rid, mol_id=r.mol_id, psi_intp=r.psi_intp, mmtrx=r.mmtrx, e1=r.e1,
                        nval=r.nval, qp_bands=r.qp_bands, polynomial=r.polynomial, niter=r.niter,
                        nen=r.nen, deltae=r.deltae, arrival=r.arrival)


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_alone_equals_in_mix(requests, precision):
    alone = []
    for r in requests:
        srv = SigmaServer(workers=1, precision=precision)
        rr = _clone(r)
        srv.run([rr], realtime=False)
        srv.close()
        alone.append(rr)
    mix = [_clone(r) for r in requests] + [_clone(r) for r in requests]
    for i, r in enumerate(mix):
        r.rid = i
    srv = SigmaServer(workers=6, precision=precision)   # all six at once
    st = srv.run(mix, realtime=False)
    srv.close()
    assert st["requests"] == 6
    for r in mix:
        a = alone[r.mol_id - 21]
        # same kernels, same tile choice, same summation order: identical bits
        assert np.array_equal(r.sigma, a.sigma), (r.rid, np.max(np.abs(r.sigma - a.sigma)))
        assert np.array_equal(r.eqp, a.eqp)


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_footprint_bounds_session_bytes(requests, precision):
    """The admission estimate is an upper bound of what the session holds
    (``ngw_session_bytes``) after serving the request, and the server's
    accounting holds the measured bytes of its idle worker."""
    for r in requests:
        srv = SigmaServer(workers=1, precision=precision)
        rr = _clone(r)
        srv.run([rr], realtime=False)
        measured = srv.sessions[0].device_bytes
        assert srv.held[0] == measured > 0
        assert rr.footprint_bytes() >= measured, (r.rid, rr.footprint_bytes(), measured)
        srv.close()


@pytest.mark.parametrize("mode", ["branches", "grouped"])
def test_grouped_small_requests_within_1mev(requests, mode, monkeypatch):
    """Small requests admitted together run as one batch -- graph branches,
    or grouped GEMM launches across their molecules (64-wide tiles) with
    NGW_BATCH_MODE=grouped; each QP energy within 1 meV of the same request
    served alone on its tuned tiles."""
    monkeypatch.setenv("NGW_BATCH_MODE", mode)
    if mode == "grouped":
        monkeypatch.setenv("NGW_DENSE", "0")    # the factored p(C) that grouped launches run
    alone = {}
    for r in requests:
        srv = SigmaServer(workers=1, precision="mixed")
        rr = _clone(r)
        srv.run([rr], realtime=False)
        srv.close()
        alone[r.mol_id] = rr.eqp
    mix = [_clone(r) for r in requests]
    srv = SigmaServer(workers=3, precision="mixed", group_work=1e30)
    st = srv.run(mix, realtime=False)
    groups = srv.groups
    srv.close()
    assert st["requests"] == 3 and groups == 1
    for r in mix:
        err = np.abs(r.eqp - alone[r.mol_id]) * 1e3
        assert np.all(err < 1.0), (r.rid, err)
