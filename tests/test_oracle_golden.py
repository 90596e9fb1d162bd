"""The oracle pinned against the reference's own golden vectors (CPU)."""
import os

import numpy as np

from oracle import fxc as ofxc
from oracle import lanczos as L

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def test_lanczos_golden_table_h_aux():
    """shared/test_lanczos/H_aux_v0.txt: notebook table with niter=5, i.e. 4
    Lanczos levels of the production recurrence (lanczos_spectra_lowcomsym.F90)."""
    d = np.load(os.path.join(GOLD, "lanczos_h_aux.npz"))
    H, v0, tab = d["H"], d["v0"], d["table"]
    levels = int(d["niter"]) - 1
    z = tab[:, 0]
    s, a, b = L.dense_lanczos_spectra(H, v0, z + 1j * float(d["eta"]), levels)
    s0, _, _ = L.dense_lanczos_spectra(H, v0, np.zeros(1, complex), levels)
    # the table is printed with 8 decimals
    assert np.max(np.abs(s0.real - tab[:, 1])) < 1e-8
    assert np.max(np.abs(s.real - tab[:, 2])) < 5e-7
    assert np.max(np.abs(s.imag - tab[:, 3])) < 5e-7
    # one more level visibly disagrees: the table really is 4 levels
    s5, _, _ = L.dense_lanczos_spectra(H, v0, z + 0.1j, levels + 1)
    assert np.max(np.abs(s5.real - tab[:, 2])) > 1e-2


def test_lda_fxc_against_libxc_testsuite():
    """f_x + f_c against LIB/libxc/testsuite/lda_x.data and lda_c_pz.data:
    unpolarised f = (v2rhoa2 + 2 v2rhoab + v2rhob2) / 4 at rho = rhoa + rhob."""
    d = np.load(os.path.join(GOLD, "libxc_lda.npz"))
    for name, fn in (("lda_x", ofxc.fx), ("lda_c_pz", ofxc.fc_pz)):
        t = d[name]
        # unpolarised points at molecular densities; above ~1e2 bohr^-3 libxc's own
        # finite difference (delta_rho = 1e-8, lda.c:153-182) loses digits
        sel = np.isclose(t[:, 0], t[:, 1]) & (t[:, 0] > 1e-6) & (t[:, 0] < 50.0)
        rho = t[sel, 0] + t[sel, 1]
        ref = (t[sel, 5] + 2.0 * t[sel, 6] + t[sel, 7]) / 4.0
        got = fn(rho)
        rel = np.abs(got - ref) / np.abs(ref)
        tol = 1e-9 if name == "lda_x" else 1e-6    # FD of PZ (delta 1e-8) vs the table's analytic values
        assert rel.max() < tol, (name, rel.max())
        # energy density as a check of the parametrisation itself
        if name == "lda_x":
            eps, _ = ofxc.ex_vx(rho)
        else:
            eps, _ = ofxc.ec_vc_pz(rho)
        assert np.max(np.abs(eps * rho - t[sel, 2]) / np.abs(t[sel, 2])) < 1e-9
        assert sel.sum() >= 5
