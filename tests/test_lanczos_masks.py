"""Oracle: per-chain Lanczos lengths and the convergence exit of the
single-vector reference routine (shared/lanczos_spectra.f90:57-58), on small
dense operators (CPU)."""
import numpy as np

from oracle import lanczos as L


def _spd(n, seed):
    rng = np.random.default_rng(seed)
    q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    lam = np.sort(rng.uniform(0.5, 4.0, n))
    return q, lam, (q * lam) @ q.T


def test_lengths_match_single_chain_runs():
    _, _, h = _spd(40, 1)
    rng = np.random.default_rng(2)
    v0 = rng.standard_normal((40, 5))
    nrm = np.linalg.norm(v0, axis=0)
    lengths = np.array([3, 8, 12, 5, 12])
    a, b, leff = L.lanczos_recurrence(lambda x: h @ x, v0, nrm, 12, lengths=lengths,
                                      return_lengths=True)
    assert np.array_equal(leff, lengths)
    for j, n in enumerate(lengths):
        aj, bj = L.lanczos_recurrence(lambda x: h @ x, v0[:, [j]], nrm[j], int(n))
        np.testing.assert_allclose(a[:n, j], aj[:, 0], rtol=1e-12, atol=0)
        np.testing.assert_allclose(b[:n, j], bj[:, 0], rtol=1e-12, atol=0)
        assert np.all(a[n:, j] == 0.0) and np.all(b[n:, j] == 0.0)
    zz = np.linspace(0.0, 5.0, 7) + 0.05j
    s = L.continued_fraction(a, b, np.repeat(zz[:, None], 5, 1), lengths=leff)
    for j, n in enumerate(lengths):
        aj, bj = L.lanczos_recurrence(lambda x: h @ x, v0[:, [j]], nrm[j], int(n))
        sj = L.continued_fraction(aj, bj, zz[:, None])[:, 0]
        np.testing.assert_allclose(s[:, j], sj, rtol=1e-12)


def test_exit_on_invariant_subspace_gives_exact_resolvent():
    q, lam, h = _spd(30, 3)
    w = np.array([0.7, -0.4, 0.25])
    v0 = q[:, [4, 11, 20]] @ w           # lies in a 3-dimensional invariant subspace
    nrm = np.linalg.norm(v0)
    a, b, leff = L.lanczos_recurrence(lambda x: h @ x, v0[:, None], nrm, 10, early_exit_eps=1e-8,
                                      return_lengths=True)
    assert leff[0] == 3
    assert abs(b[3, 0]) < 1e-8 and np.all(a[3:, 0] == 0.0) and np.all(b[4:, 0] == 0.0)
    zz = np.linspace(0.0, 5.0, 9) + 0.03j
    s = L.continued_fraction(a, b, zz[:, None], lengths=leff)[:, 0]
    exact = sum(wi * wi / (zz - li) for wi, li in zip(w, lam[[4, 11, 20]])) / (w @ w)
    np.testing.assert_allclose(s, exact, rtol=1e-10)
