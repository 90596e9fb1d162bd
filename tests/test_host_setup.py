"""CPU tests of the library's host-side setup against the oracle (bit-exact
where the reference's output is integer) and of the C ABI's exports."""
import ctypes
import os
import re

import numpy as np
import pytest

from nanogw_b200 import host, pipeline, polyfit, synth
from nanogw_b200.api import lowcomsym_pairs, sqrt_r
from oracle import cvt as ocvt
from oracle import isdf as oisdf
from oracle import pairs as opairs
from oracle import polyfit as opoly

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_exports_every_header_symbol():
    from nanogw_b200 import _lib
    L = ctypes.CDLL(_lib.LIB_PATH)
    hdr = open(os.path.join(ROOT, "include", "ngw_b200.h")).read()
    names = set(re.findall(r"^\s*(?:int|void|const char|long long|void \*)\s*\*?\s*(ngw_\w+)\s*\(", hdr, re.M))
    assert len(names) >= 20
    for n in names:
        assert hasattr(L, n), n
    assert set(_lib.SIGNATURES) <= names | {"ngw_version"}


def test_shell_sort_matches_oracle_with_ties():
    rng = np.random.default_rng(0)
    for n in (0, 1, 2, 7, 100, 1001):
        a = rng.integers(0, 5, n).astype(float)          # many ties: order of equals matters
        assert np.array_equal(host.shell_sort(a), ocvt.shell_sort(a))
        b = rng.standard_normal(n)
        p = host.shell_sort(b)
        assert np.array_equal(p, ocvt.shell_sort(b))
        assert np.all(np.diff(b[p - 1]) >= 0)


def test_cvt_and_dedup_bit_exact_small():
    mol = synth.make_molecule(4, 2.0, 5.0, 0.5, 8, 24, 5, order_fn=ocvt.shell_sort)
    init = synth.cvt_initial_points(mol.grid, 80, 5)
    a = host.cvt(mol.grid, mol.rho, init, 200)
    b = ocvt.cvt(mol.grid, mol.rho, init, 200)
    assert a[2] == b[2]
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    # forced duplicates in density: de-dup must drop the same points
    rho = mol.rho.copy()
    rho[a[0][1] - 1] = rho[a[0][0] - 1]
    assert np.array_equal(host.dedup_points(a[0], rho), ocvt.dedup_points(a[0], rho))
    assert len(host.dedup_points(a[0], rho)) == len(a[0]) - 1


def test_pair_orders():
    assert np.array_equal(lowcomsym_pairs(5, 12), opairs.lowcomsym_pairs(5, 12))
    irep = np.ones(12, dtype=int)
    prod = np.ones((1, 1), dtype=int)
    assert np.array_equal(opairs.rep_pairs(irep, 5, prod, 1), lowcomsym_pairs(5, 12))
    e1 = np.linspace(-1, 1, 12)
    cv = lowcomsym_pairs(5, 12)
    assert np.allclose(sqrt_r(e1, cv) ** 2, e1[cv[:, 1] - 1] - e1[cv[:, 0] - 1])
    pm, reps, inv = opairs.pair_maps(irep, 4, 12, prod)
    assert pm[2, 7] == 2 * 12 + 8 and len(inv[1]) == 48


def test_polyfit_matches_oracle():
    e1 = np.sort(np.r_[np.random.default_rng(1).uniform(-1.5, -0.5, 20),
                       np.random.default_rng(2).uniform(-0.3, 1.0, 60)])
    p, emin, emax = polyfit.sigma_polynomial(e1, 20, 80, 12)
    q, emin2, emax2, _ = opoly.sigma_polynomial(e1, 20, 80, 12)
    assert emin == emin2 and emax == emax2
    assert np.array_equal(p, q)


def test_isdf_fit_matches_oracle():
    mol = synth.make_molecule(4, 2.0, 5.0, 0.5, 8, 24, 5, order_fn=ocvt.shell_sort)
    intp = ocvt.dedup_points(ocvt.cvt(mol.grid, mol.rho, synth.cvt_initial_points(mol.grid, 80, 5), 200)[0],
                             mol.rho)
    psi_intp = mol.psi[intp - 1, :]
    z = pipeline.isdf_fit(mol.psi, psi_intp, 9, mol.nmem)
    zr = oisdf.isdf_fit(mol.psi, psi_intp, np.arange(1, 10), np.arange(1, mol.nmem + 1))
    assert np.max(np.abs(z - zr)) / np.max(np.abs(zr)) < 1e-10
    # the fit reproduces the pair densities at the interpolation points exactly
    assert np.max(np.abs(z[intp - 1, :] - np.eye(len(intp)))) < 1e-8
    assert pipeline.fft_box_size(9.0, 0.35) == 104 and pipeline.fft_box_size(16.0, 0.3) == 214


def test_abi_reports_errors_without_device():
    from nanogw_b200 import _lib
    L = _lib.lib()
    h = ctypes.c_void_p()
    rc = L.ngw_session_create(999, ctypes.byref(h))
    assert rc != 0 and not h.value
    assert L.ngw_last_error()


@pytest.mark.parametrize("nocc,nemp_factor", [(8, 4), (20, 3), (48, 4), (96, 4), (140, 4), (160, 4)])
def test_product_polynomial_equals_oracle_sweep(nocc, nemp_factor):
    """The product's polynomial (the reference's nx = 20..300 sweep, last
    candidate with error below 1e3) equals the oracle's bit for bit at the
    batched and serving sizes."""
    from nanogw_b200.polyfit import sigma_polynomial as product
    from oracle.polyfit import sigma_polynomial as reference
    rng = np.random.default_rng(nocc)
    e1 = np.sort(np.concatenate([rng.uniform(-0.75, -0.25, nocc),
                                 rng.uniform(-0.15, 0.5, nemp_factor * nocc)])) * 2.0
    p, emin, emax, nx = product(e1, nocc, len(e1), 12, return_nx=True)
    q, qmin, qmax, _ = reference(e1, nocc, len(e1), 12)
    assert (emin, emax) == (qmin, qmax)
    assert np.array_equal(p, q)
