"""Oracle: quasiparticle Newton solve on a cubic spline of Sigma (test
infrastructure only).

Restates ``SIGMA/spline.f90:1-77``, ``SIGMA/splint.f90``,
``SIGMA/spline_evaluate.f90:13-51``, ``SIGMA/newtonr.f90:18-58`` and the
QP part of ``SIGMA/printsigma.F90:97-130``.  Energies in eV.
"""
import numpy as np

HUGE = 1.0e10
DELTAX = 1.0e-2


def spline(xx, yy, yp1, ypn):
    """Second derivatives of a natural/clamped cubic spline for real and
    imaginary parts separately (``SIGMA/spline.f90``)."""
    nn = len(xx)
    y2 = np.zeros(nn, dtype=np.complex128)
    out = []
    for part in (lambda z: z.real, lambda z: z.imag):
        y = part(np.asarray(yy))
        d1 = part(np.complex128(yp1))
        dn = part(np.complex128(ypn))
        y2r = np.zeros(nn)
        uu = np.zeros(nn)
        if abs(d1) > HUGE:
            y2r[0] = 0.0
            uu[0] = 0.0
        else:
            y2r[0] = -0.5
            uu[0] = (3.0 / (xx[1] - xx[0])) * ((y[1] - y[0]) / (xx[1] - xx[0]) - d1)
        for i in range(1, nn - 1):
            sig = (xx[i] - xx[i - 1]) / (xx[i + 1] - xx[i - 1])
            p = sig * y2r[i - 1] + 2.0
            y2r[i] = (sig - 1.0) / p
            uu[i] = (6.0 * ((y[i + 1] - y[i]) / (xx[i + 1] - xx[i])
                            - (y[i] - y[i - 1]) / (xx[i] - xx[i - 1]))
                     / (xx[i + 1] - xx[i - 1]) - sig * uu[i - 1]) / p
        if dn > HUGE:
            qn = 0.0
            un = 0.0
        else:
            qn = 0.5
            un = (3.0 / (xx[nn - 1] - xx[nn - 2])) * (dn - (y[nn - 1] - y[nn - 2]) / (xx[nn - 1] - xx[nn - 2]))
        y2r[nn - 1] = (un - qn * uu[nn - 2]) / (qn * y2r[nn - 2] + 1.0)
        for k in range(nn - 2, -1, -1):
            y2r[k] = y2r[k] * y2r[k + 1] + uu[k]
        out.append(y2r)
    y2 = out[0] + 1j * out[1]
    return y2


def splint(xx, yy, y2a, x0):
    """Cubic spline evaluation with bisection (``SIGMA/splint.f90``)."""
    nn = len(xx)
    klo = 0
    khi = nn - 1
    while khi - klo > 1:
        k = (khi + klo + 2) // 2 - 1   # Fortran (khi+klo)/2 on 1-based indices
        if xx[k] > x0:
            khi = k
        else:
            klo = k
    hh = xx[khi] - xx[klo]
    if hh == 0.0:
        raise ValueError("bad xx input in splint")
    aa = (xx[khi] - x0) / hh
    bb = (x0 - xx[klo]) / hh
    return aa * yy[klo] + bb * yy[khi] + ((aa ** 3 - aa) * y2a[klo] + (bb ** 3 - bb) * y2a[khi]) * (hh ** 2) / 6.0


def spline_evaluate(xtable, ftable, xx):
    """f(xx) and Re f'(xx) by a spline through the interior points
    (``SIGMA/spline_evaluate.f90:37-48``)."""
    nt = len(xtable)
    yp1 = (ftable[1] - ftable[0]) / (xtable[1] - xtable[0])
    ypn = (ftable[nt - 1] - ftable[nt - 2]) / (xtable[nt - 1] - xtable[nt - 2])
    xs = xtable[1:nt - 1]
    fs = ftable[1:nt - 1]
    y2 = spline(xs, fs, yp1, ypn)
    fx = splint(xs, fs, y2, xx)
    ym = splint(xs, fs, y2, xx - DELTAX)
    yp = splint(xs, fs, y2, xx + DELTAX)
    df = (yp - ym).real / DELTAX * 0.5
    return fx, df


def newtonr(xtable, ftable, x0, xacc, max_it=20):
    """Newton-Raphson root of Re f (``SIGMA/newtonr.f90:18-58``).
    Returns (x, f(x), ierr)."""
    x = x0
    for jj in range(1, max_it + 1):
        fx, df = spline_evaluate(xtable, ftable, x)
        dx = fx.real / df
        x = x - dx
        if abs(dx) < xacc:
            fx, df = spline_evaluate(xtable, ftable, x)
            return x, fx, 0
    return x, fx, max_it


def qp_solve(sigma_c_ev, e_dft_ev, e1_ev, deltae_ev, sigx_ev, vxc_ev, xacc=0.01, sig_g_ev=None):
    """One QP state: ``SIGMA/printsigma.F90:97-125``.

    sigma_c_ev: (nen,) complex Sigma_c table on the energy grid centred on e1.
    Returns (eqp, zfac, ierr).  ``xacc`` = EN_ACC = 0.01 eV in the reference
    (printsigma.F90:60); tests use a tighter value for meV comparisons.
    """
    nen = len(sigma_c_ev)
    ii = np.arange(nen)
    xtable = e1_ev - deltae_ev * 0.5 + deltae_ev / float(nen - 1) * ii
    sg = 0.0 if sig_g_ev is None else sig_g_ev
    ftable = sigx_ev + sigma_c_ev + sg - vxc_ev + e_dft_ev - xtable
    eqp, fx, ierr = newtonr(xtable, ftable, e1_ev, xacc)
    _, d = spline_evaluate(xtable, ftable, eqp)
    zfac = -1.0 / d
    return eqp, zfac, ierr
