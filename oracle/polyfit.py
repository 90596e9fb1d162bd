"""Oracle: least-squares polynomial fit of sqrt(x) (test infrastructure only).

Restates ``shared/polyfitcheb.f90:1-96`` / ``shared/polyfit.f90:1-90`` and the
candidate sweep of ``SIGMA/calculate_sigma_lanczos_lowcomsym.F90z:252-271``.
The normal equations are solved with LAPACK ``dgesvx`` (``fact='E'``), as
``shared/linear_solver.f90:20-29`` does, through scipy's LAPACK binding.
"""
import numpy as np
from scipy.linalg import lapack


def _lsq_sqrt(xx, npoly):
    yy = np.sqrt(xx)
    nx = len(xx)
    pxx = np.ones((nx, npoly + 1))
    for ip in range(1, npoly + 1):
        pxx[:, ip] = xx ** ip
    m = pxx.T @ pxx                      # dgemm('t','n') polyfitcheb.f90:54
    y = pxx.T @ yy                       # dgemv('t')      polyfitcheb.f90:60
    res = lapack.dgesvx(m, y[:, None], fact="E")
    beta = np.array(res[7][:, 0])
    return beta


def _fit_error(beta, xmin, xmax, mx=2000):
    """Mean relative error on ``mx`` uniform points (polyfitcheb.f90:84-94)."""
    err = 0.0
    for ix in range(mx):
        tx = xmin + ix * (xmax - xmin) / (mx - 1)
        tp = 1.0
        fy = 0.0
        for ip in range(len(beta)):
            fy = fy + tp * beta[ip]
            if ip < len(beta) - 1:
                tp = tp * tx
        err = err + abs((np.sqrt(tx) - fy) / np.sqrt(tx)) / mx
    return err


def _check_range(xmin, xmax):
    if xmin >= xmax:
        xmin, xmax = xmax, xmin
    if xmin <= 0.0:
        raise ValueError("emin is smaller than zero!")
    if xmin <= 1e-4:
        raise ValueError("Polyfit_sqrt xmin is too small")
    return xmin, xmax


def polyfitcheb_sqrt(xmin, xmax, npoly, nx):
    """Fit on ``nx`` Chebyshev nodes; returns (beta low->high, fit_error)."""
    xmin, xmax = _check_range(xmin, xmax)
    emid = 0.5 * (xmin + xmax)
    scal = 0.5 * (xmax - xmin)
    dx = np.pi / (nx - 1)
    xx = emid - scal * np.cos(dx * np.arange(nx))
    beta = _lsq_sqrt(xx, npoly)
    return beta, _fit_error(beta, xmin, xmax)


def polyfit_sqrt(xmin, xmax, npoly, nx):
    """Fit on ``nx`` uniform nodes (shared/polyfit.f90:35-43)."""
    xmin, xmax = _check_range(xmin, xmax)
    dx = (xmax - xmin) / (nx - 1)
    xx = xmin + dx * np.arange(nx)
    beta = _lsq_sqrt(xx, npoly)
    return beta, _fit_error(beta, xmin, xmax)


def sigma_polynomial(e1, nval, maxicc, npoly):
    """Coefficients high->low used by the Lanczos Sigma driver.

    ``calculate_sigma_lanczos_lowcomsym.F90z:254-268``: emin/emax from the
    gap and band width; the nx = 20..300 sweep keeps the LAST candidate whose
    error is below 1e3 because ``max_fit_error`` is never updated.
    e1: KS energies (Ry, 0-based array of band 1..nmem); nval, maxicc: counts.
    Returns (polynomial high->low, emin, emax, fit_error).
    """
    emin = (e1[nval] - e1[nval - 1]) ** 2.0 / 1.25
    emax = (e1[maxicc - 1] - e1[0]) ** 2.0 * 1.25
    poly = None
    err_sel = None
    for nx in range(20, 301, 20):
        beta, err = polyfitcheb_sqrt(emin, emax, npoly, nx)
        if err < 1.0e3:
            poly = beta[::-1].copy()
            err_sel = err
    return poly, emin, emax, err_sel
