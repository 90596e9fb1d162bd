"""Host-side polynomial p(x) ~ sqrt(x) used by the Lanczos driver.

Follows ``shared/polyfitcheb.f90``: least squares on Chebyshev-spaced nodes of
[xmin, xmax] via the normal equations, solved by LAPACK ``dgesvx`` with
equilibration (``shared/linear_solver.f90:20-29``), and the mean relative
error on 2000 uniform points (``polyfitcheb.f90:84-94``).  The driver's node
sweep (``SIGMA/calculate_sigma_lanczos_lowcomsym.F90z:259-268``) tries
nx = 20, 40, ..., 300 and keeps the LAST candidate whose error is below 1e3,
because its best-error tracker is never updated; that rule is kept so the
coefficients are the reference's for every molecule.
"""
import numpy as np
from scipy.linalg import lapack


def fit_sqrt_cheb_nodes(xmin, xmax, npoly, nx):
    """Coefficients low -> high of the least-squares fit on nx Chebyshev nodes."""
    if xmin >= xmax:
        xmin, xmax = xmax, xmin
    if xmin <= 0.0:
        raise ValueError("emin is smaller than zero!")
    if xmin <= 1e-4:
        raise ValueError("Polyfit_sqrt xmin is too small")
    mid = 0.5 * (xmin + xmax)
    half = 0.5 * (xmax - xmin)
    nodes = mid - half * np.cos(np.pi / (nx - 1) * np.arange(nx))
    V = np.empty((nx, npoly + 1))
    V[:, 0] = 1.0
    for p in range(1, npoly + 1):
        V[:, p] = nodes ** p
    gram = V.T @ V
    rhs = V.T @ np.sqrt(nodes)
    out = lapack.dgesvx(gram, rhs[:, None], fact="E")
    return np.array(out[7][:, 0])          # low -> high


def fit_error(beta, xmin, xmax, mx=2000):
    """Mean relative error of the fit on mx uniform points: each point's value
    is accumulated term by term as the Fortran loop does, and the per-point
    errors are summed in point order (a sequential cumulative sum)."""
    if xmin >= xmax:
        xmin, xmax = xmax, xmin
    tx = xmin + np.arange(mx) * (xmax - xmin) / (mx - 1)
    tp = np.ones(mx)
    fy = np.zeros(mx)
    n = len(beta)
    for ip in range(n):
        fy = fy + tp * beta[ip]
        if ip < n - 1:
            tp = tp * tx
    terms = np.abs((np.sqrt(tx) - fy) / np.sqrt(tx)) / float(mx)
    return float(np.cumsum(terms)[-1])


def sigma_polynomial(e1, nval, maxicc, npoly, return_nx=False):
    """Coefficients high -> low and the fit range (emin, emax) for KS energies e1 (Ry)."""
    emin = (e1[nval] - e1[nval - 1]) ** 2.0 / 1.25
    emax = (e1[maxicc - 1] - e1[0]) ** 2.0 * 1.25
    beta, nx_sel = None, None
    for nx in range(20, 301, 20):
        b = fit_sqrt_cheb_nodes(emin, emax, npoly, nx)
        if fit_error(b, emin, emax) < 1.0e3:
            beta, nx_sel = b, nx
    if beta is None:
        raise ValueError("no polynomial fit with relative error below 1e3")
    if return_nx:
        return beta[::-1].copy(), emin, emax, nx_sel
    return beta[::-1].copy(), emin, emax
