"""Host logic of the continuous-batching loop (no GPU): admission by memory
budget, routing to the worker holding the molecule, latency accounting."""
import threading
import time

import numpy as np

from nanogw_b200.serving import SigmaRequest, SigmaServer


def _req(rid, mol, arrival, n=64, nmem=24, nval=6):
    return SigmaRequest(rid=rid, mol_id=mol, psi_intp=np.zeros((n, nmem)), mmtrx=np.zeros((n, n)),
                        e1=np.arange(nmem, dtype=float), nval=nval, qp_bands=np.array([nval, nval + 1]),
                        polynomial=np.array([1.0, 0.0]), niter=4, nen=8, arrival=arrival)


def test_budget_limits_concurrency():
    active = [0]
    peak = [0]
    lock = threading.Lock()

    def solver(w, req):
        with lock:
            active[0] += 1
            peak[0] = max(peak[0], active[0])
        time.sleep(0.05)
        with lock:
            active[0] -= 1
        req.eqp = np.zeros(len(req.qp_bands))

    reqs = [_req(i, i % 3, 0.0) for i in range(6)]
    one = reqs[0].footprint_bytes()
    srv = SigmaServer(workers=4, hbm_budget_gb=2.5 * one / (1 << 30), solver=solver)
    st = srv.run(reqs, realtime=False)
    assert st["requests"] == 6 and st["solves"] == 12
    assert peak[0] == 2                      # the budget holds two at a time
    assert srv.peak_used <= 2.5 * one
    assert all(r.finish >= r.start >= 0 for r in reqs)


def test_arrivals_respected_and_routing():
    order = []

    def solver(w, req):
        order.append((req.rid, w))
        time.sleep(0.01)

    reqs = [_req(0, 7, 0.0), _req(1, 7, 0.08), _req(2, 8, 0.0)]
    srv = SigmaServer(workers=2, solver=solver)
    st = srv.run(reqs, realtime=True)
    assert reqs[1].start >= 0.08 - 1e-3      # not admitted before it arrives
    # request 1 reuses the worker that already holds molecule 7
    assert reqs[1].worker == reqs[0].worker
    assert st["p99_ms"] >= st["p50_ms"] > 0


def test_oversize_request_refused_with_budget_error():
    from nanogw_b200._lib import NGW_ERR_BUDGET
    ran = []

    def solver(w, req):
        ran.append(req.rid)

    small = _req(0, 1, 0.0)
    big = _req(1, 2, 0.0, n=512, nmem=200, nval=40)
    srv = SigmaServer(workers=2, hbm_budget_gb=1.5 * small.footprint_bytes() / (1 << 30), solver=solver)
    assert big.footprint_bytes() > srv.budget
    st = srv.run([small, big], realtime=False)     # nothing in flight when `big` is considered
    assert ran == [0]
    assert st["refused"] == 1 and st["requests"] == 1
    assert big.error is not None and big.error.code == NGW_ERR_BUDGET


def test_idle_resident_memory_counts_and_is_released():
    """Memory an idle worker's session still holds (measured, as
    ngw_session_bytes reports it) counts against the budget; when a new
    request does not fit, idle sessions other than the chosen worker are
    emptied first."""
    held = {}

    def solver(w, req):
        held[w] = req.footprint_bytes()      # the session keeps what it used
        time.sleep(0.01)

    def session_bytes(w):
        return held.get(w, 0)

    reqs = [_req(i, 10 + i, 0.0) for i in range(3)]
    one = reqs[0].footprint_bytes()
    srv = SigmaServer(workers=3, hbm_budget_gb=2.5 * one / (1 << 30), solver=solver,
                      session_bytes=session_bytes)
    orig_release = srv.release

    def release(w):
        held[w] = 0
        orig_release(w)
    srv.release = release
    st = srv.run(reqs, realtime=False)
    assert st["requests"] == 3 and st["refused"] == 0
    assert srv.released >= 1                 # an idle session gave its memory back
    assert srv.peak_used <= srv.budget
    assert sum(srv.held) <= srv.budget


def test_largest_first_policy_orders_admission():
    order = []

    def solver(w, req):
        order.append(req.rid)
        time.sleep(0.01)

    reqs = [_req(0, 1, 0.0, n=32), _req(1, 2, 0.0, n=128), _req(2, 3, 0.0, n=64)]
    srv = SigmaServer(workers=1, solver=solver)
    srv.run(reqs, realtime=False, policy="largest")
    assert order == [1, 2, 0]
    order.clear()
    srv.run([_req(0, 1, 0.0, n=32), _req(1, 2, 0.0, n=128), _req(2, 3, 0.0, n=64)], realtime=False)
    assert order == [0, 1, 2]


def test_small_requests_grouped():
    """With group_work set, small waiting requests are admitted together
    (one free worker each) and run as one group; large ones alone."""
    seen = []

    def solver(w, req):
        seen.append((req.rid, w))
        time.sleep(0.01)

    reqs = [_req(0, 1, 0.0, n=32), _req(1, 2, 0.0, n=32), _req(2, 3, 0.0, n=256), _req(3, 4, 0.0, n=32)]
    small = reqs[0].work()
    srv = SigmaServer(workers=4, solver=solver, group_work=2.0 * small, group_max=8)
    srv.precision = "mixed"
    st = srv.run(reqs, realtime=False)
    assert st["requests"] == 4
    assert srv.groups == 1
    assert len({w for _, w in seen}) == 4          # every request on its own worker
    grouped = [r for r in reqs if r.rid in (0, 1, 3)]
    assert len({round(r.start, 3) for r in grouped}) == 1   # admitted together


def _req_sized(nval, nmem, n, nqp, npoly=12):
    return SigmaRequest(rid=0, mol_id=0, psi_intp=np.zeros((n, nmem)), mmtrx=np.zeros((n, n)),
                        e1=np.arange(nmem, dtype=float), nval=nval,
                        qp_bands=np.arange(nval - nqp // 2, nval - nqp // 2 + nqp) + 1,
                        polynomial=np.ones(npoly + 1), niter=150, nen=400)


def test_dense_form_memory_counts_in_mixed_footprint():
    # 12-atom class (N_cv = 2700, 600 ISDF points, 720 chains): the library
    # forms H = p(C) here, so the mixed footprint holds H in split BF16 and
    # the FP64 formation's eight N_cv^2 matrices
    small = _req_sized(30, 120, 600, 6)
    dense = small.dense_bytes()
    n2 = small.ncv ** 2
    assert dense >= 4 * n2 + 8 * 8 * n2
    assert small.footprint_bytes(mixed=True) - small.footprint_bytes(mixed=False) == dense
    # above N_cv = 16384 the library never takes the dense form
    big = _req_sized(80, 400, 640, 4)
    assert big.ncv > 16384 and big.dense_bytes() == 0
    # a degree-1 polynomial (TDA-like) has no dense form either
    assert _req_sized(30, 120, 600, 6, npoly=1).dense_bytes() == 0


def test_fp64_server_admits_without_dense_memory():
    req = _req_sized(30, 120, 600, 6)
    budget_gb = (req.footprint_bytes(mixed=False) + (1 << 20)) / (1 << 30)
    assert req.footprint_bytes(mixed=True) > budget_gb * (1 << 30)
    ran = []

    def solver(w, r):
        ran.append(r.rid)
        r.eqp = np.zeros(len(r.qp_bands))

    st = SigmaServer(workers=1, precision="fp64", hbm_budget_gb=budget_gb, solver=solver).run([req],
                                                                                                realtime=False)
    assert ran == [0] and st["refused"] == 0
    st = SigmaServer(workers=1, precision="mixed", hbm_budget_gb=budget_gb, solver=solver).run([req],
                                                                                                 realtime=False)
    assert st["refused"] == 1
