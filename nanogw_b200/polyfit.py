"""Host-side polynomial p(x) ~ sqrt(x) used by the Lanczos driver.

Follows ``shared/polyfitcheb.f90``: least squares on Chebyshev-spaced nodes of
[xmin, xmax] via the normal equations, solved by LAPACK ``dgesvx`` with
equilibration (``shared/linear_solver.f90:20-29``).  The driver's node sweep
(``SIGMA/calculate_sigma_lanczos_lowcomsym.F90z:259-268``) keeps the last
candidate (nx = 300) because its best-error tracker is never updated; that
behaviour is kept so coefficients match the reference's.
"""
import numpy as np
from scipy.linalg import lapack


def fit_sqrt_cheb_nodes(xmin, xmax, npoly, nx):
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


def sigma_polynomial(e1, nval, maxicc, npoly):
    """Coefficients high -> low and the fit range (emin, emax) for KS energies e1 (Ry)."""
    emin = (e1[nval] - e1[nval - 1]) ** 2.0 / 1.25
    emax = (e1[maxicc - 1] - e1[0]) ** 2.0 * 1.25
    beta = fit_sqrt_cheb_nodes(emin, emax, npoly, 300)
    return beta[::-1].copy(), emin, emax
