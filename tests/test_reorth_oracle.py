"""Full reorthogonalisation of the Lanczos chains in the oracle (CPU): in
exact arithmetic it leaves alpha/beta unchanged, so over the first steps
(before rounding has grown) they equal the reference recurrence's; over a
long run the reorthogonalised recurrence is insensitive to rounding noise
(its own spread under 1e-15 perturbations stays tiny) while the reference
recurrence's grows to O(1)."""
import numpy as np

from oracle import lanczos as L
from oracle import sigma as OS


def _start(S, nb=6):
    p, pn2 = OS.start_vectors(S.psi_intp, S.M, S.Cmtrx, S.sqrtR, S.nval, np.arange(1, nb + 1))
    return p, np.sqrt(pn2)


def _ab(S, p, pn, niter, reorth, perturb=0.0):
    zz = np.repeat(np.array([0.1 + 0.02j])[:, None], p.shape[1], 1)
    _, a, b = L.lanczos_spectra_isdf(p, pn, zz, niter, S.poly, S.Cmtrx, S.M, S.sqrtR, perturb=perturb,
                                     reorth=reorth)
    return a, b


def test_reorth_equals_reference_before_rounding_grows(small_system):
    """Over the first steps the two recurrences agree to the reference
    recurrence's own rounding spread (the degree-12 Horner polynomial
    amplifies rounding ~4e5 times, so that spread is ~1e-10 from step 3)."""
    S = small_system
    p, pn = _start(S)
    a0, b0 = _ab(S, p, pn, 6, False)
    a1, b1 = _ab(S, p, pn, 6, True)
    ap, bp = _ab(S, p, pn, 6, False, perturb=1e-15)
    spread = np.max(np.abs(ap - a0) / np.abs(a0), axis=1)
    err = np.max(np.abs(a1 - a0) / np.abs(a0), axis=1)
    assert err[0] == 0.0                     # a_0 comes before any Gram-Schmidt step
    assert np.all(err <= np.maximum(1e-9, 100.0 * spread)), (err, spread)
    errb = np.max(np.abs(b1[1:] - b0[1:]) / np.abs(b0[1:]), axis=1)
    assert np.all(errb < 1e-8), errb


def test_reorth_is_stable_under_rounding_noise(small_system):
    S = small_system
    p, pn = _start(S)
    niter = 60
    a_r, _ = _ab(S, p, pn, niter, True)
    a_p, _ = _ab(S, p, pn, niter, True, perturb=1e-15)
    spread_reorth = np.max(np.abs(a_p - a_r) / np.abs(a_r))
    a0, _ = _ab(S, p, pn, niter, False)
    a0p, _ = _ab(S, p, pn, niter, False, perturb=1e-15)
    spread_ref = np.max(np.abs(a0p - a0) / np.abs(a0))
    assert spread_reorth < 1e-9, spread_reorth
    assert spread_ref > 1e3 * spread_reorth, (spread_ref, spread_reorth)
