"""Oracle: ISDF Casida matvec, Horner polynomial matvec, Lanczos recurrence and
continued fraction (FP64 numpy).  Test infrastructure only.

Vectors are stored Fortran-style column blocks ``vec(ncv, blksz)``: numpy arrays
of shape ``(ncv, blksz)``.
"""
import numpy as np


def matvec_isdf(vec, cmtrx, mmtrx, sqrtR, tamm_d=False):
    """H x for a block of columns.

    Follows ``shared/apply_matvec_lowcomsym.F90:112-128`` (R^1/2 scaling),
    ``:228-229`` (C x), ``:283-284`` (M (C x)), ``:365-366`` (C^T ...) and
    ``:396-412`` (diagonal combine):
        non-TDA: H x = R^{3/2} (R^{1/2} x) + 4 R^{1/2} C^T M C R^{1/2} x
        TDA:     A x = R x + 2 C^T M C x
    cmtrx: (n_isdf, ncv) pair products, mmtrx: (n_isdf, n_isdf), sqrtR: (ncv,).
    """
    vec = np.asarray(vec, dtype=np.float64)
    one_d = vec.ndim == 1
    if one_d:
        vec = vec[:, None]
    s = sqrtR[:, None]
    if tamm_d:
        h = vec.copy()
    else:
        h = s * vec
    tmp = cmtrx @ h                      # (n_isdf, blksz)
    mc = mmtrx @ tmp                     # (n_isdf, blksz)
    cmc = cmtrx.T @ mc                   # (ncv, blksz)
    if tamm_d:
        h = (s * s) * h
        h = h + 2.0 * cmc
    else:
        h = (s * s * s) * h
        h = h + 4.0 * s * cmc
    return h[:, 0] if one_d else h


def polynomial_matvec_isdf(vec, polynomial, cmtrx, mmtrx, sqrtR, matvec=None):
    """p(H) x by Horner's rule, coefficients stored high->low
    (``polynomial(1) = a_n``).  Follows
    ``shared/apply_matvec_lowcomsym.F90:490-514`` (and ``shared/apply_matvec.f90:169-184``).
    ``matvec`` overrides the H application (used to inject rounding-size noise).
    """
    npoly = len(polynomial) - 1
    hold = np.array(vec, dtype=np.float64, copy=True)
    hvec = None
    for k in range(1, npoly + 1):
        hvec = matvec(hold) if matvec else matvec_isdf(hold, cmtrx, mmtrx, sqrtR)
        if k == 1:
            hvec = polynomial[0] * hvec + polynomial[1] * vec
        else:
            hvec = hvec + polynomial[k] * vec
        hold = hvec
    return hvec


def _gram_schmidt_twice(basis, w, sel, k):
    """w -= V (V^T w) with V the chains' vectors v_0 .. v_k (basis:
    (blksz, niter + 1, ncv); w: (ncv, len(sel))), repeated once for the
    chains whose pass shrank ||w|| below 1/sqrt(2) of its value ("twice is
    enough": Daniel, Gragg, Kaufman and Stewart, Math. Comp. 30 (1976))."""
    Vs = basis[:, : k + 1, :] if len(sel) == basis.shape[0] else basis[sel, : k + 1, :]
    before = np.einsum("ij,ij->j", w, w)
    again = np.ones(w.shape[1], dtype=bool)
    for _ in range(2):
        idx = np.nonzero(again)[0]
        if len(idx) == 0:
            break
        V = Vs[idx]
        h = np.matmul(V, w[:, idx].T[:, :, None])                # (n, k+1, 1)
        w[:, idx] = w[:, idx] - np.matmul(V.transpose(0, 2, 1), h)[:, :, 0].T
        after = np.einsum("ij,ij->j", w[:, idx], w[:, idx])
        again[idx] = after < 0.5 * before[idx]
        before[idx] = after
    return w


def lanczos_recurrence(apply_h, v0, v0_norm, niter, early_exit_eps=None, lengths=None,
                       return_lengths=False, reorth=False):
    """Lanczos alpha/beta for a block of independent chains.

    Follows ``shared/lanczos_spectra_lowcomsym.F90:67-166`` exactly (no
    reorthogonalisation; ``b(1) = 1``; the ``k+1 <= niter`` guard).
    ``lengths`` (optional, per chain) runs chain j for lengths[j] steps: the
    same loop with niter = lengths[j].  With ``early_exit_eps`` a chain stops
    at the top of step k when ``|b_k| < eps``, as the single-vector routine
    does (``shared/lanczos_spectra.f90:57-58``); the tail the reference leaves
    uninitialised is zero here and the chain's effective length is k.
    ``reorth`` (not in the reference): after ``w -= a_k v_k`` every chain's w
    is orthogonalised against its v_0 .. v_k by classical Gram-Schmidt applied
    twice, before ``b_{k+1} = ||w||``.
    Returns (a, b) with shape (niter, blksz) [, effective lengths].
    """
    v0 = np.asarray(v0, dtype=np.float64)
    if v0.ndim == 1:
        v0 = v0[:, None]
    blksz = v0.shape[1]
    v0_norm = np.broadcast_to(np.asarray(v0_norm, dtype=np.float64), (blksz,))
    L = np.full(blksz, niter) if lengths is None else np.clip(np.asarray(lengths), 1, niter)
    leff = L.copy()
    a = np.zeros((niter, blksz))
    b = np.zeros((niter, blksz))
    vec = v0 / v0_norm[None, :]
    b[0, :] = 1.0
    basis = None
    if reorth:
        basis = np.zeros((blksz, niter + 1, v0.shape[0]))
        basis[:, 0, :] = vec.T
    wvec = apply_h(vec)
    a[0] = np.einsum("ij,ij->j", wvec, vec)
    wvec = wvec - a[0][None, :] * vec
    if reorth:
        wvec = _gram_schmidt_twice(basis, wvec, np.arange(blksz), 0)
    if niter >= 2:
        b[1] = np.where(L >= 2, np.sqrt(np.einsum("ij,ij->j", wvec, wvec)), 0.0)
    for k in range(1, niter):
        act = k < leff
        if early_exit_eps is not None:
            stop = act & (np.abs(b[k]) < early_exit_eps)
            leff[stop] = k
            act &= ~stop
        sel = np.nonzero(act)[0]
        if len(sel) == 0:
            break
        w = wvec[:, sel] / b[k, sel][None, :]
        v = -vec[:, sel] * b[k, sel][None, :]
        v, w = w, v
        if reorth:
            basis[sel, k, :] = v.T
        w = w + apply_h(v)
        a[k, sel] = np.einsum("ij,ij->j", w, v)
        more = k + 1 < L[sel]
        if more.any():
            w[:, more] = w[:, more] - a[k, sel][more][None, :] * v[:, more]
            if reorth:
                w[:, more] = _gram_schmidt_twice(basis, w[:, more], sel[more], k)
            b[k + 1, sel[more]] = np.sqrt(np.einsum("ij,ij->j", w[:, more], w[:, more]))
        vec[:, sel] = v
        wvec[:, sel] = w
    if return_lengths:
        return a, b, leff
    return a, b


def continued_fraction(a, b, zz, lengths=None):
    """S(z) = <v|(z-H)^-1|v> from the Lanczos coefficients.

    Follows ``shared/lanczos_spectra_lowcomsym.F90:175-188``:
    S = 0; for j = niter..1: S = (j==1 ? 1 : b_j^2) / (z - a_j - S).
    ``lengths`` (optional): chain j uses its first lengths[j] coefficients.
    a, b: (niter, blksz); zz: (nz, blksz) complex.  Returns (nz, blksz).
    """
    a = np.asarray(a)
    b = np.asarray(b)
    if a.ndim == 1:
        a = a[:, None]
        b = b[:, None]
    zz = np.asarray(zz, dtype=np.complex128)
    if zz.ndim == 1:
        zz = zz[:, None]
    niter = a.shape[0]
    s = np.zeros(np.broadcast_shapes(zz.shape, (1, a.shape[1])), dtype=np.complex128)
    for j in range(niter - 1, -1, -1):
        num = 1.0 if j == 0 else b[j] * b[j]
        with np.errstate(divide="ignore", invalid="ignore"):   # masked-out tails may divide 0/0
            nxt = num / (zz - a[j][None, :] - s)
        s = nxt if lengths is None else np.where((j < np.asarray(lengths))[None, :], nxt, s)
    return s


def perturbed(apply_h, rel, seed=1):
    """Wrap an operator so every product carries a relative rounding-size
    perturbation ``rel``.  Used to measure how sensitive the unreorthogonalised
    recurrence is to rounding: two FP64 codes that are equal in exact
    arithmetic differ by about this much per matvec."""
    rng = np.random.default_rng(seed)

    def f(x):
        y = apply_h(x)
        return y * (1.0 + rel * rng.standard_normal(y.shape))
    return f


def lanczos_spectra_isdf(v0, v0_norm, zz, niter, polynomial, cmtrx, mmtrx, sqrtR,
                         tamm_d=False, perturb=0.0, lengths=None, early_exit_eps=None,
                         return_lengths=False, reorth=False):
    """``lanczos_spectra_isdf_lowcomsym`` (``shared/lanczos_spectra_lowcomsym.F90:7-190``):
    the spectra <P|1/(zz-p(H))|P> for a block of start vectors; per-chain
    lengths and the single-vector form's exit (``shared/lanczos_spectra.f90:57-58``)
    as in ``lanczos_recurrence``.  Returns (spectra (nz, blksz), a, b[, lengths])."""
    mv = lambda x: matvec_isdf(x, cmtrx, mmtrx, sqrtR, tamm_d=tamm_d)   # noqa: E731
    if perturb:
        mv = perturbed(mv, perturb)
    if tamm_d:
        apply_h = mv
    else:
        def apply_h(x):
            return polynomial_matvec_isdf(x, polynomial, cmtrx, mmtrx, sqrtR, matvec=mv)
    a, b, leff = lanczos_recurrence(apply_h, v0, v0_norm, niter, early_exit_eps=early_exit_eps,
                                    lengths=lengths, return_lengths=True, reorth=reorth)
    spec = continued_fraction(a, b, zz, lengths=leff)
    if return_lengths:
        return spec, a, b, leff
    return spec, a, b


def dense_lanczos_spectra(H, v0, zz, niter):
    """The dense-matrix test driver of ``shared/test_lanczos/test_lanczos.f90``
    with the production recurrence (``niter`` Lanczos levels) -- used to pin the
    oracle against the reference's golden table ``H_aux_v0.txt``."""
    v0 = np.asarray(v0, dtype=np.float64)
    nrm = np.sqrt(v0 @ v0)
    a, b = lanczos_recurrence(lambda x: H @ x, v0[:, None], nrm, niter)
    return continued_fraction(a, b, np.asarray(zz)[:, None])[:, 0], a[:, 0], b[:, 0]
