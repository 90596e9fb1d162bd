"""Oracle: ISDF fit, FFT-Poisson and the ISDF kernel matrices (test
infrastructure only).

* ``isdf_fit``       -- ``shared/isdf_parallel_sym_UltraLowMem.F90:439-667``
                        (P, Q, P_intp, Q_intp, A = P_intp*Q_intp,
                        B = P*Q, solve A Z = B, zeta = Z^T), C1 symmetry.
* ``fft_box_size``   -- ``shared/parsec_wfn.F90:365-381``
                        (nfft = even(nint(4*rmax/h)); adjust_fft is a no-op
                        without ESSL, ``shared/fft_module.F90z:1507-1551``).
* ``coulomb_0d``     -- ``shared/fft_module.F90z:628-691`` (truncated Coulomb,
                        trunc = 2*rmax, ``shared/parsec_wfn.F90:421-425``).
* ``poisson``        -- ``shared/fft_module.F90z:122-177``.
* ``kernel_mmtrx``   -- ``shared/isdf_parallel_sym_UltraLowMem.F90:805-889``
                        (norm_factor = ntrans/hcub, ``:312``).
* ``k_integrate``    -- ``shared/k_integrate_isdf.F90z:243-348``.
FFTW is an external library of the reference and is not pinned by any
reference test; numpy's FFT is used here (parity to tolerance).
"""
import numpy as np

QZERO = 1.0e-8   # any value below the smallest nonzero |G|^2 gives the same table


def isdf_fit(psi, psi_intp, vbands, cbands):
    """zeta (ngrid, n_isdf).

    psi: (ngrid, nmem) orbitals on the grid; psi_intp: (n_isdf, nmem) at the
    interpolation points; vbands/cbands: 1-based band lists summed in P and Q
    (``ivlist``/``iclist``)."""
    v = np.asarray(vbands) - 1
    c = np.asarray(cbands) - 1
    P = psi_intp[:, v] @ psi[:, v].T            # (n_isdf, ngrid)
    Q = psi_intp[:, c] @ psi[:, c].T
    P_i = psi_intp[:, v] @ psi_intp[:, v].T     # (n_isdf, n_isdf)
    Q_i = psi_intp[:, c] @ psi_intp[:, c].T
    A = P_i * Q_i
    B = P * Q
    Z = np.linalg.solve(A, B)                   # pdgesv
    return Z.T.copy()


def fft_box_size(rmax, h):
    n = int(np.rint(4.0 * rmax / h))
    if n % 2:
        n += 1
    return n


def coulomb_0d(nfft, h, trunc):
    """Truncated Coulomb kernel on the full (n, n, n) FFT grid in numpy's
    frequency order: 8*pi*(1-cos(trunc*|G|))/|G|^2, 8*pi*trunc^2/2 at G=0."""
    L = nfft * h
    b = 2.0 * np.pi / L
    j = np.fft.fftfreq(nfft, d=1.0 / nfft)
    g2 = (b * j)[:, None, None] ** 2 + (b * j)[None, :, None] ** 2 + (b * j)[None, None, :] ** 2
    v = np.empty_like(g2)
    small = g2 < QZERO * QZERO
    v[small] = trunc ** 2 / 2.0
    gs = g2[~small]
    v[~small] = (1.0 - np.cos(trunc * np.sqrt(gs))) / gs
    return 8.0 * np.pi * v


def poisson(rho_cols, grid_idx, nfft, vcoul, workers=None):
    """v_c * rho for each column: pack on the box, FFT, multiply, FFT back,
    unpack, scale by 1/N^3 (the inverse transform already divides).
    rho_cols: (ngrid, ncol); grid_idx: (ngrid, 3) integer coordinates.
    ``workers``: threads for scipy's FFT (None: numpy's single-threaded FFT);
    both are pocketfft and agree to rounding."""
    out = np.empty_like(rho_cols)
    ix = np.mod(grid_idx, nfft)
    vh = vcoul[:, :, : nfft // 2 + 1]
    if workers is None:
        fwd = np.fft.rfftn
        inv = lambda f: np.fft.irfftn(f, s=(nfft, nfft, nfft), axes=(0, 1, 2))   # noqa: E731
    else:
        import scipy.fft as sfft
        fwd = lambda b: sfft.rfftn(b, workers=workers)                                # noqa: E731
        inv = lambda f: sfft.irfftn(f, s=(nfft, nfft, nfft), workers=workers)         # noqa: E731
    for k in range(rho_cols.shape[1]):
        box = np.zeros((nfft, nfft, nfft))
        box[ix[:, 0], ix[:, 1], ix[:, 2]] = rho_cols[:, k]
        f = fwd(box)
        f *= vh
        r = inv(f)
        out[:, k] = r[ix[:, 0], ix[:, 1], ix[:, 2]]
    return out


def kernel_mmtrx(zeta, vzeta, hcub, ntrans=1, fxc=None):
    """(M_C, M_xc): norm * zeta^T (v_c zeta), norm * zeta^T (f_xc * zeta)."""
    nf = 1.0 / hcub * ntrans
    mc = nf * (zeta.T @ vzeta)
    mxc = None
    if fxc is not None:
        mxc = nf * (zeta.T @ (fxc[:, None] * zeta))
    return mc, mxc


def k_integrate(psi_intp, mc, mxc, rows, cols, kflag=0):
    """K(m1m2; m3m4) = (psi_m1 psi_m2)^T (M) (psi_m3 psi_m4) with
    M = [kflag<2] M_C + [kflag>0] M_xc.  rows/cols: (n, 2) 1-based band pairs.
    Returns (len(rows), len(cols))."""
    M = np.zeros_like(mc)
    if kflag < 2:
        M = M + mc
    if kflag > 0:
        M = M + mxc
    r = np.asarray(rows) - 1
    c = np.asarray(cols) - 1
    cr = psi_intp[:, r[:, 0]] * psi_intp[:, r[:, 1]]
    cc = psi_intp[:, c[:, 0]] * psi_intp[:, c[:, 1]]
    tmp = M @ cr
    return tmp.T @ cc
