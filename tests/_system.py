"""Small deterministic ISDF system shared by the tests: a 4-atom synthetic
molecule on a 5-bohr sphere (h = 0.5), 8 occupied + 24 empty orbitals, 96 ISDF
points; the Coulomb kernel comes from the oracle's numpy FFT-Poisson so CPU
tests and GPU parity tests see identical inputs."""
import functools

import numpy as np

from nanogw_b200 import synth
from nanogw_b200.api import lowcomsym_pairs, sqrt_r
from oracle import cvt as ocvt
from oracle import isdf as oisdf
from oracle import polyfit as opoly


class System:
    pass


@functools.lru_cache(maxsize=4)
def make_small_system(seed=3, n_atoms=4, R=5.0, h=0.5, nocc=8, nemp=24, n_isdf=96, npoly=12):
    mol = synth.make_molecule(n_atoms, 2.0, R, h, nocc, nemp, seed, order_fn=ocvt.shell_sort)
    init = synth.cvt_initial_points(mol.grid, n_isdf, seed)
    intp, _, iters = ocvt.cvt(mol.grid, mol.rho, init, 1000)
    intp = ocvt.dedup_points(intp, mol.rho)
    psi_intp = np.asfortranarray(mol.psi[intp - 1, :])
    nmem = mol.nmem
    zeta = oisdf.isdf_fit(mol.psi, psi_intp, np.arange(1, nocc + 2), np.arange(1, nmem + 1))
    nfft = oisdf.fft_box_size(R, h)
    vc = oisdf.coulomb_0d(nfft, h, 2.0 * R)
    vz = oisdf.poisson(zeta, mol.grid_idx, nfft, vc)
    M, _ = oisdf.kernel_mmtrx(zeta, vz, mol.hcub)
    s = System()
    s.mol = mol
    s.psi_intp = psi_intp
    s.M = np.asfortranarray(M)
    s.e1 = mol.e1.copy()
    s.nval = nocc
    s.nmem = nmem
    s.cvpair = lowcomsym_pairs(nocc, nmem)
    s.sqrtR = sqrt_r(s.e1, s.cvpair)
    s.Cmtrx = s.psi_intp[:, s.cvpair[:, 1] - 1] * s.psi_intp[:, s.cvpair[:, 0] - 1]
    s.poly, s.emin, s.emax, _ = opoly.sigma_polynomial(s.e1, nocc, nmem, npoly)
    s.zeta = zeta
    s.nfft = nfft
    s.intp = intp
    s.cvt_iters = iters
    return s
