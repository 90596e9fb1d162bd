"""Setup pipeline: molecule -> ISDF points -> Psi_intp, zeta -> Coulomb kernel M.

Order follows ``SIGMA/sigma.F90:318-738``: CVT point selection on the
density (``shared/cvt.F90``; iterations on the device, bit-identical to the
host restatement), density de-duplication (``sigma.F90:377-461``),
the ISDF fit of the interpolation vectors zeta
(``shared/isdf_parallel_sym_UltraLowMem.F90:439-667``) and the Coulomb block
``M = ntrans/hcub zeta^T v_c zeta`` built on the device
(``:687-889``; library entry ``ngw_build_coulomb_kernel``).
The fit (P, Q products and the A zeta^T = B solve) runs on the device by
default (``ngw_build_isdf_kernel``; zeta stays in HBM and feeds the Poisson
build directly); ``device_fit=False`` keeps the numpy fit (host LAPACK) for
machines without a GPU.
"""
from dataclasses import dataclass

import numpy as np

from . import host, synth
from .api import lowcomsym_pairs, sqrt_r


@dataclass
class IsdfOperator:
    psi_intp: np.ndarray     # (n_isdf, nmem)
    mmtrx: np.ndarray        # (n_isdf, n_isdf) Coulomb block, Ry
    intp: np.ndarray         # 1-based grid indices of the points
    e1: np.ndarray           # (nmem,) Ry
    nval: int
    cvt_iters: int
    zeta: np.ndarray = None
    mxc: np.ndarray = None   # f_xc block (n_isdf, n_isdf), Ry, when built

    @property
    def nmem(self):
        return self.psi_intp.shape[1]

    @property
    def n_isdf(self):
        return self.psi_intp.shape[0]

    def pairs(self):
        cv = lowcomsym_pairs(self.nval, self.nmem)
        return cv, sqrt_r(self.e1, cv)


def fft_box_size(rmax, h):
    """nfft = even(nint(4 rmax / h)) (``shared/parsec_wfn.F90:365-381``)."""
    n = int(np.rint(4.0 * rmax / h))
    return n + (n % 2)


def isdf_fit(psi, psi_intp, mv, nmem):
    """zeta (ngrid, n_isdf): P = sum_{v<=mv} psi_v(r_mu) psi_v(r),
    Q = sum_{c<=nmem} psi_c(r_mu) psi_c(r), A = P_intp*Q_intp, B = P*Q, A Z = B."""
    pv = psi_intp[:, :mv]
    pc = psi_intp[:, :nmem]
    P = pv @ psi[:, :mv].T
    Q = pc @ psi[:, :nmem].T
    A = (pv @ pv.T) * (pc @ pc.T)
    B = P * Q
    del P, Q
    Z = np.linalg.solve(A, B)
    return np.ascontiguousarray(Z.T)


def build_operator(mol, n_isdf, session, qp_bands=(), seed=0, max_cvt_iter=100000,
                   keep_zeta=False, device_fit=True, with_fxc=False):
    grid = mol.grid
    init = synth.cvt_initial_points(grid, n_isdf, seed if seed else mol.seed)
    # CVT iterations on the session's device (bit-identical to the host form)
    intp, _, iters = host.cvt(grid, mol.rho, init, max_cvt_iter, session=session if device_fit else None)
    intp = host.dedup_points(intp, mol.rho)
    mv = max([mol.nval] + [int(b) for b in qp_bands])
    nfft = fft_box_size(mol.rmax, mol.h)
    mxc = None
    if device_fit and not keep_zeta:
        psi_intp, M, mxc = session.build_isdf_kernel(mol.psi, mol.grid_idx, intp, mv, nfft, mol.h,
                                                     2.0 * mol.rmax, mol.rho if with_fxc else None)
        zeta = None
    else:
        psi_intp = np.asfortranarray(mol.psi[intp - 1, :])
        zeta = isdf_fit(mol.psi, psi_intp, mv, mol.nmem)
        M = session.build_coulomb_kernel(zeta, mol.grid_idx, nfft, mol.h, 2.0 * mol.rmax)
        if with_fxc:
            mxc = session.build_fxc_kernel(zeta, mol.rho, mol.h)
    op = IsdfOperator(psi_intp=psi_intp, mmtrx=np.asfortranarray(M), intp=intp, e1=mol.e1.copy(),
                      nval=mol.nval, cvt_iters=iters, zeta=zeta if keep_zeta else None, mxc=mxc)
    return op


def exchange_and_vxc(mol, session, qp_bands):
    """Diagonal Sigma_x and V_xc (Ry) of the QP bands on the device
    (``ngw_fock_exchange``, ``ngw_vxc_matrix``): closed shell, occupation 1 per
    spin for the nval lowest bands, truncated Coulomb radius 2 rmax."""
    occ = np.zeros(mol.nmem)
    occ[: mol.nval] = 1.0
    qp = np.asarray(qp_bands, dtype=np.int32)
    nfft = fft_box_size(mol.rmax, mol.h)
    kx = session.fock_exchange(mol.psi, mol.grid_idx, nfft, mol.h, 2.0 * mol.rmax, occ, qp)
    vxc, _ = session.vxc_matrix(mol.psi, mol.rho, qp)
    return np.diag(kx).copy(), np.diag(vxc).copy()


def qp_bands_near_gap(nval, nqp):
    """The nqp bands nearest the gap: nqp/2 highest occupied, the rest lowest empty."""
    nocc = nqp // 2
    return np.array(list(range(nval - nocc + 1, nval + 1)) +
                    list(range(nval + 1, nval + 1 + nqp - nocc)), dtype=np.int32)
