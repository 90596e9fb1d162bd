"""Oracle for Sigma_x and V_xc (CPU): the LDA potentials against libxc's own
test tables, and structural properties of the exchange matrix."""
import os

import numpy as np

from oracle import exchange as OX

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_lda_potentials_against_libxc_testsuite():
    """v_x and v_c (Ry) = 2 x libxc's vrho (Ha) at unpolarised points of
    LIB/libxc/testsuite/lda_x.data and lda_c_pz.data."""
    d = np.load(os.path.join(GOLD, "libxc_lda.npz"))
    for k, name in enumerate(("lda_x", "lda_c_pz")):
        t = d[name]
        sel = np.isclose(t[:, 0], t[:, 1]) & (t[:, 0] > 1e-6)
        rho = t[sel, 0] + t[sel, 1]
        v = OX.lda_potentials(rho)[k] / 2.0
        rel = np.abs(v - t[sel, 3]) / np.abs(t[sel, 3])
        assert rel.max() < 1e-9, (name, rel.max())


def test_exchange_matrix_is_symmetric_negative_semidefinite(small_system):
    """K_x = -sum_n occ_n G_n with G_n the Gram matrix of the pair densities
    psi_n psi_m under the (non-negative) truncated Coulomb kernel: symmetric
    and negative semidefinite; the diagonal of occupied states is negative."""
    S = small_system
    mol = S.mol
    occ = np.zeros(S.nmem)
    occ[: S.nval] = 1.0
    bands = np.array([S.nval - 2, S.nval - 1, S.nval, S.nval + 1, S.nval + 3])
    kx = OX.fock_exchange(mol.psi, mol.grid_idx, S.nfft, mol.h, 2.0 * mol.rmax, occ, bands)
    assert np.array_equal(kx, kx.T)
    w = np.linalg.eigvalsh(kx)
    assert w.max() < 1e-10 * np.abs(w).max()
    assert np.all(np.diag(kx)[:3] < 0.0)


def test_vxc_matrix_diagonal_is_the_expectation(small_system):
    S = small_system
    mol = S.mol
    bands = np.array([1, S.nval, S.nval + 1])
    vxc, vx = OX.vxc_matrix(mol.psi, mol.rho, bands)
    vxr, vcr = OX.lda_potentials(mol.rho)
    for i, m in enumerate(bands):
        p = mol.psi[:, m - 1]
        assert np.isclose(vxc[i, i], np.sum(p * p * (vxr + vcr)), rtol=1e-12)
        assert np.isclose(vx[i, i], np.sum(p * p * vxr), rtol=1e-12)
    assert np.all(np.diag(vxc) < 0.0)
