"""Continuous-batching request loop for Sigma_c solves.

Requests (one molecule's ISDF operator + the QP states to solve) arrive over
time; the server keeps a pool of workers, each a library session with its own
CUDA stream, cuBLAS handle, graph cache and device-resident state (orbitals at
the ISDF points, Coulomb kernel, pair products, split-BF16 operands, deflated
eigenpairs, Lanczos vectors).  A request is admitted when a worker is free and
the device memory it needs fits the budget next to everything already
resident; it is routed to a worker that already holds its molecule when one is
free (the operator then stays resident and is not re-uploaded).  Requests on
different workers run concurrently on the device -- a new request starts as
soon as a slot frees, it does not wait for a batch to form.

Admission accounting: every worker's session keeps device memory between
requests (operator, split-BF16 operands, eigenpairs, chain buffers); that
memory counts against the budget whether the worker is busy or idle, measured
with ``ngw_session_bytes`` once a request is done.  A request about to run
reserves its footprint estimate (an upper bound of what the session will hold
while serving it) on the worker it is routed to.  When the budget is short,
idle workers other than the chosen one give their memory back (their session
is recreated empty).  A request whose footprint alone exceeds the budget is
refused with ``NGW_ERR_BUDGET`` and never runs.

Latency = finish - arrival; throughput = QP states solved per second.
"""
import heapq
import threading
import time
from dataclasses import dataclass, field

import numpy as np

from ._lib import NGW_ERR_BUDGET, NGWError
from .api import RYD, Session


@dataclass
class SigmaRequest:
    rid: int
    mol_id: int
    psi_intp: np.ndarray
    mmtrx: np.ndarray
    e1: np.ndarray
    nval: int
    qp_bands: np.ndarray
    polynomial: np.ndarray
    niter: int = 150
    nen: int = 400
    deltae: float = 4.0
    ecuts: float = 0.02
    sigx_ev: float = -12.0
    vxc_ev: float = -10.0
    arrival: float = 0.0
    # filled in by the server
    start: float = field(default=0.0)
    finish: float = field(default=0.0)
    worker: int = field(default=-1)
    sigma: np.ndarray = field(default=None)
    eqp: np.ndarray = field(default=None)
    error: Exception = field(default=None)

    @property
    def nmem(self):
        return self.psi_intp.shape[1]

    @property
    def ncv(self):
        return self.nval * (self.nmem - self.nval)

    def work(self):
        """Matvec work of the request (chain-steps x the operator's size), the
        ordering key of the largest-first policy."""
        n = self.psi_intp.shape[0]
        return float(len(self.qp_bands)) * self.nmem * self.niter * n * (2.0 * self.ncv + n)

    def footprint_bytes(self, mixed=True):
        """Device memory the request needs: operator (FP64 + split-BF16 +
        pair products), Lanczos / Clenshaw state of all its chains and, in
        mixed precision where the library may take the dense p(C) form, that
        form's memory."""
        n, ncv, nb = self.psi_intp.shape[0], self.ncv, len(self.qp_bands) * self.nmem
        op = 8 * (n * self.nmem + n * n + n * ncv) + 2 * 2 * 2 * (n + 64) * (ncv + 128)
        chains = nb * ncv * (8 * 6 + 4 * 3 + 2 * 2) + nb * self.niter * 16 + nb * (self.nen + 1) * 16
        dense = self.dense_bytes() if mixed else 0
        return int(op + chains + dense + (96 << 20))

    def dense_bytes(self):
        """Peak device memory of the dense p(C) form when the library may
        choose it for this request (mixed precision), else 0.

        The library (``want_dense`` in csrc/abi.cu) takes the dense form for
        N_cv <= 16384 when forming H = p(C) once plus one N_cv x N_cv product
        per Lanczos step costs less than the factored form's 2p GEMMs per
        step.  Here the test runs with the formation already paid and the
        most deflated pairs the plan asks for (64), the case that favours
        the dense form most, so the estimate stays an upper bound.  Memory:
        H in split BF16 (kept in the session, 4 B per padded element) and
        the FP64 formation's temporaries, freed after it (the Casida matrix,
        the Paterson-Stockmeyer powers T_0 .. T_m, two Horner accumulators,
        M C_isdf and the rank-k deflation products)."""
        n, ncv, nb = self.psi_intp.shape[0], self.ncv, len(self.qp_bands) * self.nmem
        p = len(self.polynomial) - 1
        if ncv > 16384 or p < 2:
            return 0
        kdef = 64
        dense_step = 3.0 * 2.0 * ncv * ncv * nb / 0.9e15 + 10e-6
        fact_step = p * (3.0 * 4.0 * (n + kdef) * ncv * nb / 0.6e15 + 10e-6)
        if dense_step >= fact_step:
            return 0
        m = max(2, int(np.ceil(np.sqrt(p + 1.0))))
        powers = m + 1
        cv_pad = -(-ncv // 128) * 128
        kpad = -(-ncv // 64) * 64
        resident = 2 * 2 * cv_pad * kpad
        formation = 8 * ncv * ncv * (1 + powers + 2) + 8 * n * ncv + 8 * (2 * ncv * kdef + kdef * kdef)
        return int(resident + formation)


class SigmaServer:
    def __init__(self, device=0, workers=2, precision="mixed", hbm_budget_gb=150.0, solver=None,
                 session_bytes=None, group_work=0.0, group_max=8):
        """`solver(worker, request)` replaces the device solve and
        `session_bytes(worker)` the device-memory query (host-logic tests).

        group_work > 0 (mixed precision): a waiting request whose matvec work
        (``SigmaRequest.work``) is at most group_work is admitted together with
        up to group_max - 1 other such waiting requests, one free worker each,
        and the group runs as one batch (``sigma_lanczos_batch``; its form
        follows NGW_BATCH_MODE: graph branches by default, grouped GEMM
        launches across the molecules with ``grouped``)."""
        self.group_work = float(group_work) if precision == "mixed" else 0.0
        self.group_max = max(1, int(group_max))
        self.groups = 0                           # groups of two or more requests run
        self.device = device
        self.precision = precision
        self.budget = int(hbm_budget_gb * (1 << 30))
        self.solver = solver
        self._session_bytes = session_bytes
        self.sessions = [] if solver else [Session(device, precision) for _ in range(workers)]
        self.nworkers = workers
        self.resident = [None] * workers          # mol_id held by each worker
        self.held = [0] * workers                 # device bytes each worker's session holds
        self.peak_used = 0
        self.released = 0                         # idle sessions emptied to make room

    def close(self):
        for s in self.sessions:
            s.close()

    def worker_bytes(self, w):
        """Device bytes worker w's session holds now (``ngw_session_bytes``)."""
        if self._session_bytes is not None:
            return int(self._session_bytes(w))
        if self.solver:
            return 0
        return self.sessions[w].device_bytes

    def release(self, w):
        """Give an idle worker's device memory back: its session is recreated
        empty (the autotuner's tile cache is process-wide and stays)."""
        if not self.solver:
            self.sessions[w].close()
            self.sessions[w] = Session(self.device, self.precision)
        self.resident[w] = None
        self.held[w] = 0
        self.released += 1

    def _solve(self, w, req):
        if self.solver:
            self.solver(w, req)
            self.resident[w] = req.mol_id
            return
        from .api import lowcomsym_pairs, sqrt_r
        s = self.sessions[w]
        if self.resident[w] != req.mol_id:
            s.set_isdf(req.psi_intp, req.mmtrx)
            cv = lowcomsym_pairs(req.nval, req.nmem)
            s.set_pairs(cv, sqrt_r(req.e1, cv))
            self.resident[w] = req.mol_id
        sig = s.calculate_sigma_lanczos(req.e1, req.nval, req.qp_bands, req.nen, req.deltae, req.ecuts,
                                        req.niter, req.polynomial)
        e1 = req.e1[req.qp_bands - 1] * RYD
        eqp, _, _ = s.qp_newton(sig * RYD, e1, e1, req.deltae * RYD, req.sigx_ev, req.vxc_ev)
        req.sigma = sig
        req.eqp = eqp

    def _solve_group(self, ws, reqs):
        if self.solver:
            for w, r in zip(ws, reqs):
                self._solve(w, r)
            return
        from .api import lowcomsym_pairs, sigma_lanczos_batch, sqrt_r
        for w, r in zip(ws, reqs):
            s = self.sessions[w]
            if self.resident[w] != r.mol_id:
                s.set_isdf(r.psi_intp, r.mmtrx)
                cv = lowcomsym_pairs(r.nval, r.nmem)
                s.set_pairs(cv, sqrt_r(r.e1, cv))
                self.resident[w] = r.mol_id
        sigs = sigma_lanczos_batch([self.sessions[w] for w in ws],
                                   [dict(e1=r.e1, nval=r.nval, qp_bands=r.qp_bands, nen=r.nen, deltae=r.deltae,
                                         ecuts=r.ecuts, niter=r.niter, polynomial=r.polynomial) for r in reqs])
        for w, r, sig in zip(ws, reqs, sigs):
            e1 = r.e1[r.qp_bands - 1] * RYD
            r.eqp = self.sessions[w].qp_newton(sig * RYD, e1, e1, r.deltae * RYD, r.sigx_ev, r.vxc_ev)[0]
            r.sigma = sig

    def run(self, requests, realtime=True, policy="fifo"):
        """Serve `requests` (arrival times in seconds from the start).  With
        realtime=False every request is available at t=0 (closed loop).
        Among the requests waiting for a slot, policy "fifo" admits the
        earliest arrival first and "largest" the one with the most matvec
        work first (longest-processing-time order: on a closed batch of
        uneven requests the largest no longer starts last and runs alone).
        Requests larger than the whole budget are refused (``req.error`` is
        an NGWError with code NGW_ERR_BUDGET) and counted in ``refused``."""
        if policy not in ("fifo", "largest"):
            raise ValueError("policy must be 'fifo' or 'largest'")
        reqs = sorted(requests, key=lambda r: r.arrival)
        mixed = self.precision == "mixed"     # the dense p(C) form's memory counts in mixed precision
        lock = threading.Condition()
        free = list(range(self.nworkers))
        inflight = {}
        reserved = [0] * self.nworkers
        pending = []          # arrived, not admitted: heap of (arrival, rid, req)
        t0 = time.perf_counter()
        errors = []
        refused = []

        def used():
            return sum(max(h, r) for h, r in zip(self.held, reserved))

        def worker_done(w, req):
            held = self.worker_bytes(w)
            with lock:
                req.finish = time.perf_counter() - t0
                free.append(w)
                self.held[w] = held
                reserved[w] = 0
                del inflight[req.rid]
                lock.notify_all()

        def work(w, req):
            try:
                self._solve(w, req)
            except Exception as e:       # keep serving; report at the end
                req.error = e
                errors.append((req.rid, repr(e)))
            worker_done(w, req)

        def work_group(ws, rs):
            try:
                self._solve_group(ws, rs)
            except Exception as e:
                for r in rs:
                    r.error = e
                    errors.append((r.rid, repr(e)))
            for w, r in zip(ws, rs):
                worker_done(w, r)

        threads = []
        i = 0
        with lock:
            while i < len(reqs) or pending or inflight:
                now = time.perf_counter() - t0
                while i < len(reqs) and (not realtime or reqs[i].arrival <= now):
                    key = reqs[i].arrival if policy == "fifo" else -reqs[i].work()
                    heapq.heappush(pending, (key, reqs[i].rid, reqs[i]))
                    i += 1
                admitted = False
                while pending and free:
                    _, _, req = pending[0]
                    need = req.footprint_bytes(mixed)
                    if need > self.budget:
                        heapq.heappop(pending)
                        req.error = NGWError(NGW_ERR_BUDGET, f"request {req.rid} needs {need} bytes, more "
                                                             f"than the {self.budget}-byte budget")
                        req.start = req.finish = time.perf_counter() - t0
                        refused.append(req.rid)
                        continue
                    # prefer a free worker that already holds this molecule
                    w = next((x for x in free if self.resident[x] == req.mol_id), free[0])
                    reserved[w] = need
                    if used() > self.budget:
                        # idle sessions other than w give their memory back
                        for x in free:
                            if x != w and self.held[x] > 0 and used() > self.budget:
                                self.release(x)
                    if used() > self.budget:
                        reserved[w] = 0
                        break                    # wait for memory held by running requests
                    heapq.heappop(pending)
                    free.remove(w)
                    group_w, group_r = [w], [req]
                    if self.group_work > 0 and req.work() <= self.group_work:
                        # other small waiting requests join, one free worker each
                        aside = []
                        while pending and free and len(group_r) < self.group_max:
                            item = heapq.heappop(pending)
                            r2 = item[2]
                            need2 = r2.footprint_bytes(mixed)
                            if r2.work() > self.group_work or need2 > self.budget:
                                aside.append(item)
                                continue
                            w2 = next((x for x in free if self.resident[x] == r2.mol_id), free[0])
                            reserved[w2] = need2
                            if used() > self.budget:
                                reserved[w2] = 0
                                aside.append(item)
                                break
                            free.remove(w2)
                            group_w.append(w2)
                            group_r.append(r2)
                        for item in aside:
                            heapq.heappush(pending, item)
                    self.peak_used = max(self.peak_used, used())
                    for w2, r2 in zip(group_w, group_r):
                        inflight[r2.rid] = r2
                        r2.start = time.perf_counter() - t0
                        r2.worker = w2
                    if len(group_r) > 1:
                        self.groups += 1
                        th = threading.Thread(target=work_group, args=(group_w, group_r), daemon=True)
                    else:
                        th = threading.Thread(target=work, args=(w, req), daemon=True)
                    threads.append(th)
                    th.start()
                    admitted = True
                if admitted:
                    continue
                if i < len(reqs) and realtime:
                    timeout = max(0.0, reqs[i].arrival - (time.perf_counter() - t0))
                    lock.wait(timeout=timeout if timeout > 0 else 0.0005)
                else:
                    lock.wait(timeout=0.05)
        for th in threads:
            th.join()
        wall = time.perf_counter() - t0
        if errors:
            raise RuntimeError(f"{len(errors)} requests failed, first: {errors[0]}")
        done = [r for r in reqs if r.error is None]
        lat = np.array([r.finish - r.arrival for r in done]) if done else np.zeros(1)
        solves = sum(len(r.qp_bands) for r in done)
        return {"requests": len(done), "refused": len(refused), "solves": solves, "wall_s": wall,
                "solves_per_s": solves / wall,
                "p50_ms": float(np.percentile(lat, 50) * 1e3),
                "p99_ms": float(np.percentile(lat, 99) * 1e3)}
