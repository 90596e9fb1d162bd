"""Oracle: the ISDF operator of a molecule from the oracle's own pieces
(test infrastructure only).

Follows the order of ``SIGMA/sigma.F90:318-738``: CVT point selection on the
density (``shared/cvt.F90``, C restatement in ``cvt.c``), de-duplication
(``SIGMA/sigma.F90:377-461``), the ISDF fit
(``shared/isdf_parallel_sym_UltraLowMem.F90:439-667``) with P summed over the
bands 1..max(nval, QP bands) and Q over all bands, FFT-Poisson
(``shared/fft_module.F90z:122-177``, box ``shared/parsec_wfn.F90:365-381``,
truncation radius 2 rmax) and the Coulomb block
``M = ntrans/hcub zeta^T v_c zeta`` (``:805-889``).
"""
import numpy as np

from . import cvt as ocvt
from . import isdf as oisdf


def build_operator(grid, grid_idx, psi, rho, nval, h, rmax, init_pts, qp_bands=(), fft_workers=None):
    """(psi_intp (n_isdf, nmem) Fortran order, M (n_isdf, n_isdf), intp 1-based).

    grid: (ngrid, 3) coordinates; grid_idx: integer coordinates; psi: (ngrid,
    nmem) orbitals; rho: density; init_pts: the CVT's initial centres."""
    intp, _, _ = ocvt.cvt(grid, rho, init_pts)
    intp = ocvt.dedup_points(intp, rho)
    psi_intp = np.asfortranarray(psi[intp - 1, :])
    nmem = psi.shape[1]
    mv = max([nval] + [int(b) for b in qp_bands])
    zeta = oisdf.isdf_fit(psi, psi_intp, np.arange(1, mv + 1), np.arange(1, nmem + 1))
    nfft = oisdf.fft_box_size(rmax, h)
    vc = oisdf.coulomb_0d(nfft, h, 2.0 * rmax)
    vz = oisdf.poisson(zeta, grid_idx, nfft, vc, workers=fft_workers)
    M, _ = oisdf.kernel_mmtrx(zeta, vz, h ** 3)
    return psi_intp, np.asfortranarray(M), intp
