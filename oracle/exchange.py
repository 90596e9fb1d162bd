"""Oracle: bare exchange Sigma_x and V_xc matrix elements (test
infrastructure only).

* ``fock_exchange`` restates ``SIGMA/fock_exchange.F90z:16-228`` for one spin,
  one k-point, C1 symmetry and real orbitals on a finite system (``per = 0``):
  for every pair (m2 in the Sigma bands, n <= maxv) the pair density
  psi_n psi_m2 goes through the FFT-Poisson solve with the truncated Coulomb
  kernel (``Zcreate_coul_0D``), is multiplied by psi_n and projected on every
  psi_m1 (m1 <= m2 in the band list):
      K_x(m1, m2) += -(ntrans / hcub) <psi_m1 | psi_n V_c[psi_n psi_m2]> occ_n
  with n running over 1..maxv (maxv = highest state with occ > tol_occ = 0.01,
  ``shared/myconstants.F90:51``), then K_x(m2, m1) = K_x(m1, m2).
* ``vxc_matrix`` restates ``SIGMA/vxc.F90z:147-165`` with
  ``shared/vxcmtxel.F90z``: v_x = 2 v_x^LDA(rho) and v_c = 2 (v_xc - v_x)
  (``shared/xc_module.F90:523-657,672-829``, LDA: Slater exchange and the
  Perdew-Zunger correlation potential), matrix elements
      V(m1, m2) = ntrans <psi_m1 | v | psi_m2>.
Orbitals are normalised as sum_r psi^2 ntrans = 1; energies in Rydberg.
"""
import numpy as np

from . import fxc as F
from . import isdf as I

TOL_OCC = 0.01


def fock_exchange(psi, grid_idx, nfft, h, trunc, occ, sig_bands, ntrans=1):
    """K_x (nsig, nsig) in Ry.  psi: (ngrid, nmem); occ: (nmem,);
    sig_bands: 1-based band indices (the reference's s_map order)."""
    sig = np.asarray(sig_bands)
    occ = np.asarray(occ, dtype=np.float64)
    maxv = int(np.max(np.nonzero(occ > TOL_OCC)[0]) + 1) if np.any(occ > TOL_OCC) else 0
    vc = I.coulomb_0d(nfft, h, trunc)
    fac = float(ntrans) / h ** 3
    ns = len(sig)
    kx = np.zeros((ns, ns))
    ps = psi[:, sig - 1]
    for jj in range(ns):
        m2 = sig[jj]
        rho = psi[:, :maxv] * psi[:, [m2 - 1]]            # columns n = 1..maxv
        v = I.poisson(rho, grid_idx, nfft, vc)
        w = psi[:, :maxv] * v
        g = ps[:, : jj + 1].T @ w                          # (jj+1, maxv)
        kx[: jj + 1, jj] = -(g * occ[None, :maxv]).sum(axis=1) * fac
    for jj in range(ns):
        for ii in range(jj):
            kx[jj, ii] = kx[ii, jj]
    return kx


def lda_potentials(rho):
    """(v_x, v_c) on the grid in Ry (``vx_get`` / ``vxc_get`` x 2, unpolarised)."""
    _, vx = F.ex_vx(rho)
    _, vc = F.ec_vc_pz(rho)
    return 2.0 * vx, 2.0 * vc


def vxc_matrix(psi, rho, sig_bands, ntrans=1):
    """(V_xc, V_x) matrices (nsig, nsig) in Ry."""
    sig = np.asarray(sig_bands)
    vx, vc = lda_potentials(np.asarray(rho, dtype=np.float64))
    ps = psi[:, sig - 1]
    mx = ntrans * (ps.T @ (vx[:, None] * ps))
    mc = ntrans * (ps.T @ (vc[:, None] * ps))
    return mx + mc, mx
