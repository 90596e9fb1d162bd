"""Oracle: LDA exchange-correlation kernel f_xc (test infrastructure only).

``shared/xc_module.F90:853-893`` (``fxc_get``, kflag 1/2, nspin = 1):
f_xc = 2 * (f_x + f_c)  [Ry bohr^3], with
* f_x from libxc's analytic LDA exchange (``LIB/libxc/src/lda_x.c``):
  e_x = -(3/4)(3/pi)^(1/3) rho^(4/3), v_x = (4/3) eps_x, f_x = (4/9) eps_x / rho;
* f_c by libxc's finite difference of the Perdew-Zunger potential
  (``LIB/libxc/src/lda.c:153-182``, delta_rho = 1e-8, centred unless
  rho < 2 delta_rho) with the original PZ constants (``lda_c_pz.c`` "PZ Original").
Unpolarised inputs; energies in Hartree inside, Rydberg on output.
"""
import numpy as np

PZ = dict(gamma=-0.1423, beta1=1.0529, beta2=0.3334, a=0.0311, b=-0.048, c=0.0020, d=-0.0116)


def rs_of(rho):
    return (3.0 / (4.0 * np.pi * rho)) ** (1.0 / 3.0)


def ex_vx(rho):
    eps = -0.75 * (3.0 / np.pi) ** (1.0 / 3.0) * rho ** (1.0 / 3.0)
    return eps, 4.0 / 3.0 * eps


def fx(rho):
    eps, _ = ex_vx(rho)
    return 4.0 / 9.0 * eps / rho


def ec_vc_pz(rho):
    rho = np.asarray(rho, dtype=np.float64)
    rs = rs_of(rho)
    srs = np.sqrt(rs)
    lrs = np.log(rs)
    p = PZ
    den = 1.0 + p["beta1"] * srs + p["beta2"] * rs
    ec_lo = p["gamma"] / den
    vc_lo = ec_lo * (1.0 + 7.0 / 6.0 * p["beta1"] * srs + 4.0 / 3.0 * p["beta2"] * rs) / den
    ec_hi = p["a"] * lrs + p["b"] + p["c"] * rs * lrs + p["d"] * rs
    vc_hi = (p["a"] * lrs + (p["b"] - p["a"] / 3.0) + 2.0 / 3.0 * p["c"] * rs * lrs
             + (2.0 * p["d"] - p["c"]) * rs / 3.0)
    hi = rs < 1.0
    return np.where(hi, ec_hi, ec_lo), np.where(hi, vc_hi, vc_lo)


def fc_pz(rho, delta=1e-8):
    rho = np.asarray(rho, dtype=np.float64)
    _, v1 = ec_vc_pz(rho + delta)
    fwd = rho < 2.0 * delta
    lo = np.where(fwd, rho, rho - delta)
    _, v2 = ec_vc_pz(lo)
    return np.where(fwd, (v1 - v2) / delta, (v1 - v2) / (2.0 * delta))


def fxc_lda(rho):
    """f_xc(rho) in Ry bohr^3 (``fxc_get``: (f_x + f_c) * 2)."""
    return (fx(rho) + fc_pz(rho)) * 2.0
