"""Full-size check on the 12-atom workload (71k grid points, 30 + 90 orbitals,
600 ISDF points, 150 Lanczos steps): the library's own setup pipeline (CVT,
ISDF fit, Coulomb kernel on the device), then the plain FP64 path against the
mixed-precision path.  Size-independent properties: QP energies within 1 meV
(the mixed path's bar), Sigma_c agreement away from poles, and the CVT points
bit-identical to the oracle's."""
import numpy as np
import pytest

import nanogw_b200 as ngw
from nanogw_b200 import pipeline, synth
from nanogw_b200.polyfit import sigma_polynomial

pytestmark = pytest.mark.gpu

RYD = 13.60569193


@pytest.fixture(scope="module")
def workload():
    mol = synth.make_molecule(12, 4.0, 9.0, 0.35, 30, 90, seed=11)
    qp = pipeline.qp_bands_near_gap(mol.nval, 6)
    with ngw.Session(0) as s:
        op = pipeline.build_operator(mol, 600, s, qp_bands=qp, seed=11)
    poly, emin, emax = sigma_polynomial(op.e1, op.nval, op.nmem, 12)
    return mol, op, qp, poly


def test_fp64_vs_mixed_qp_energies(workload):
    mol, op, qp, poly = workload
    cv, sr = op.pairs()
    qsel = qp[[2, 3]]
    out = {}
    for prec in ("fp64", "mixed"):
        with ngw.Session(0, prec) as s:
            s.set_isdf(op.psi_intp, op.mmtrx)
            s.set_pairs(cv, sr)
            sig = s.calculate_sigma_lanczos(op.e1, op.nval, qsel, 400, 4.0, 0.02, 150, poly)
            e1 = op.e1[qsel - 1] * RYD
            eqp, z, ierr = s.qp_newton(sig * RYD, e1, e1, 4.0 * RYD, -12.0, -10.0, 1e-6)
            out[prec] = (sig, eqp, ierr)
    err_mev = np.abs(out["mixed"][1] - out["fp64"][1]) * 1e3
    print("QP fp64", out["fp64"][1], "mixed", out["mixed"][1], "err meV", err_mev)
    assert np.all(out["fp64"][2] == 0) and np.all(out["mixed"][2] == 0)
    assert np.all(err_mev < 1.0)


def test_cvt_points_match_oracle(workload):
    from oracle import cvt as ocvt
    mol, op, qp, poly = workload
    init = synth.cvt_initial_points(mol.grid, 600, 11)
    intp, _, _ = ocvt.cvt(mol.grid, mol.rho, init)
    intp = ocvt.dedup_points(intp, mol.rho)
    assert np.array_equal(intp, op.intp)


def test_device_cvt_bit_identical(workload):
    """ngw_cvt_device (iterations on the GPU) equals the host ngw_cvt bit for
    bit at full size: points, indices and iteration count."""
    import time
    from nanogw_b200 import host
    mol, op, qp, poly = workload
    init = synth.cvt_initial_points(mol.grid, 600, 11)
    t = time.perf_counter()
    ih, ph, nh = host.cvt(mol.grid, mol.rho, init)
    th = time.perf_counter() - t
    with ngw.Session(0) as s:
        host.cvt(mol.grid[:5000], mol.rho[:5000], init[:50], 3, session=s)   # warm the kernels
        t = time.perf_counter()
        idv, pdv, ndv = host.cvt(mol.grid, mol.rho, init, session=s)
        td = time.perf_counter() - t
    print(f"CVT host {th:.3f} s, device {td:.3f} s, {nh} iterations")
    assert nh == ndv
    assert np.array_equal(ih, idv)
    assert np.array_equal(ph, pdv)
