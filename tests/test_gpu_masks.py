"""Per-chain Lanczos lengths and convergence masks through the C ABI against
the oracle (FP64 path), and the mixed path with per-chain lengths within
1 meV.  Chains of a Sigma_c block run longest first with each step's
matvecs restricted to the chains still running; results come back in chain
order.  Tolerances as in test_gpu_parity: 1e-10 (alpha/beta) / 1e-8
(Sigma_c) or 100 x the oracle's own spread under a 1e-15 perturbation."""
import numpy as np
import pytest

import nanogw_b200 as ngw
from oracle import lanczos as L
from oracle import sigma as OS

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def sess(small_system):
    s = ngw.Session(0, "fp64")
    s.set_isdf(small_system.psi_intp, small_system.M)
    s.set_pairs(small_system.cvpair, small_system.sqrtR)
    yield s
    s.close()


def _rel(a, b):
    return np.max(np.abs(a - b)) / np.max(np.abs(b))


def test_spectra_per_chain_lengths(sess, small_system):
    S = small_system
    p, pn2 = OS.start_vectors(S.psi_intp, S.M, S.Cmtrx, S.sqrtR, S.nval, np.arange(1, 9))
    lengths = np.array([9, 4, 7, 2, 9, 5, 1, 6], dtype=np.int32)
    zz = np.repeat((np.linspace(-1.0, 1.0, 11) + 0.02j)[:, None], 8, 1)
    args = (p, np.sqrt(pn2), zz, 9, S.poly, S.Cmtrx, S.M, S.sqrtR)
    spec_r, a_r, b_r = L.lanczos_spectra_isdf(*args, lengths=lengths)
    _, a_p, _ = L.lanczos_spectra_isdf(*args, lengths=lengths, perturb=1e-15)
    spec, a, b = sess.lanczos_spectra_isdf(p, np.sqrt(pn2), zz, 9, S.poly, chain_niter=lengths)
    for j, n in enumerate(lengths):
        assert np.all(a[n:, j] == 0.0) and np.all(b[n:, j] == 0.0)
        spread = np.abs(a_p[:n, j] - a_r[:n, j]) / np.abs(a_r[:n, j])
        err = np.abs(a[:n, j] - a_r[:n, j]) / np.abs(a_r[:n, j])
        assert np.all(err <= np.maximum(1e-10, 100.0 * spread)), (j, err, spread)
    sp = _rel(L.lanczos_spectra_isdf(*args, lengths=lengths, perturb=1e-15)[0], spec_r)
    assert _rel(spec, spec_r) <= max(1e-9, 100.0 * sp)


def test_spectra_convergence_exit(sess, small_system):
    """A start vector inside a 3-dimensional invariant subspace of the
    Tamm-Dancoff operator A (no polynomial, so leakage out of the subspace
    stays at rounding level): with eps = 1e-8 (the single-vector reference
    value) the chain stops after 3 steps and the continued fraction is the
    exact three-pole resolvent."""
    S = small_system
    ncv = len(S.sqrtR)
    h = L.matvec_isdf(np.eye(ncv), S.Cmtrx, S.M, S.sqrtR, tamm_d=True)
    lam, q = np.linalg.eigh(0.5 * (h + h.T))
    idx = [ncv // 4, ncv // 2, (3 * ncv) // 4]
    w = np.array([0.6, -0.5, 0.3])
    v0 = q[:, idx] @ w
    zz = np.linspace(0.0, 2.0 * lam[-1], 13) + 0.03j
    spec, a, b = sess.lanczos_spectra_isdf(v0[:, None], np.linalg.norm(v0), zz, 10, None,
                                           tamm_d=True, early_exit_eps=1e-8)
    assert abs(b[3, 0]) < 1e-8
    assert np.all(a[3:, 0] == 0.0) and np.all(b[4:, 0] == 0.0)
    exact = sum(wi * wi / (zz - li) for wi, li in zip(w, lam[idx])) / (w @ w)
    assert _rel(spec[:, 0], exact) < 1e-9
    # the same through the oracle's exit
    ref, ar, br = L.lanczos_spectra_isdf(v0[:, None], np.linalg.norm(v0), zz[:, None], 10, None,
                                         S.Cmtrx, S.M, S.sqrtR, tamm_d=True, early_exit_eps=1e-8)
    assert np.all(ar[3:, 0] == 0.0)
    assert _rel(spec[:, 0], ref[:, 0]) < 1e-9
    # without the exit the chain runs on (lowcomsym form): all 10 alphas set
    _, a2, _ = sess.lanczos_spectra_isdf(v0[:, None], np.linalg.norm(v0), zz, 10, None, tamm_d=True)
    assert np.all(np.isfinite(a2[:3, 0]))


def _lengths(nqp, nb, niter, seed):
    return np.random.default_rng(seed).integers(4, niter + 1, size=(nqp, nb)).astype(np.int32)


def test_sigma_per_chain_lengths(sess, small_system):
    S = small_system
    qp = np.array([S.nval - 1, S.nval, S.nval + 1, S.nval + 2], dtype=np.int32)
    nen, deltae, ecuts, niter = 41, 2.0, 0.02, 16
    lens = _lengths(len(qp), S.nmem, niter, 5)
    got, a, b = sess.calculate_sigma_lanczos(S.e1, S.nval, qp, nen, deltae, ecuts, niter, S.poly,
                                             return_ab=True, chain_niter=lens)
    for i, m in enumerate(qp):
        args = (S.psi_intp, S.M, S.e1, S.nval, int(m), nen, deltae, ecuts, niter, S.poly)
        ref = OS.sigma_c_state(*args, lengths=lens[i])
        rp = OS.sigma_c_state(*args, lengths=lens[i], perturb=1e-15)
        err, spread = _rel(got[:, i], ref), _rel(rp, ref)
        assert err <= max(1e-8, 100.0 * spread), (i, err, spread)
        ai = a[:, i * S.nmem:(i + 1) * S.nmem]
        for j in range(S.nmem):
            assert np.all(ai[lens[i, j]:, j] == 0.0)


def test_sigma_uniform_lengths_bit_identical(sess, small_system):
    S = small_system
    qp = np.array([S.nval, S.nval + 1], dtype=np.int32)
    plain = sess.calculate_sigma_lanczos(S.e1, S.nval, qp, 21, 2.0, 0.02, 12, S.poly)
    full = np.full((len(qp), S.nmem), 12, dtype=np.int32)
    got = sess.calculate_sigma_lanczos(S.e1, S.nval, qp, 21, 2.0, 0.02, 12, S.poly, chain_niter=full)
    np.testing.assert_array_equal(got, plain)


def test_mixed_sigma_lengths_within_1mev(small_system):
    S = small_system
    qp = np.array([S.nval - 1, S.nval, S.nval + 1, S.nval + 2], dtype=np.int32)
    nen, deltae, ecuts, niter = 81, 2.0, 0.02, 24
    lens = _lengths(len(qp), S.nmem, niter, 7)
    with ngw.Session(0, "mixed") as m:
        m.set_isdf(S.psi_intp, S.M)
        m.set_pairs(S.cvpair, S.sqrtR)
        got = m.calculate_sigma_lanczos(S.e1, S.nval, qp, nen, deltae, ecuts, niter, S.poly,
                                        chain_niter=lens)
    refs = np.stack([OS.sigma_c_state(S.psi_intp, S.M, S.e1, S.nval, int(mm), nen, deltae, ecuts,
                                      niter, S.poly, lengths=lens[i]) for i, mm in enumerate(qp)],
                    axis=1)
    sigx = np.full(len(qp), -0.4)
    vxc = np.full(len(qp), -0.6)
    e_ref = OS.qp_energies(refs.T, S.e1, S.e1, qp, deltae, sigx, vxc, xacc_ev=1e-7)
    e_got = OS.qp_energies(got.T, S.e1, S.e1, qp, deltae, sigx, vxc, xacc_ev=1e-7)
    err_mev = np.array([abs(x[0] - y[0]) * 1e3 for x, y in zip(e_got, e_ref)])
    print("QP error (meV):", err_mev)
    assert np.all(err_mev < 1.0)
