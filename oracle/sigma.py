"""Oracle: the Lanczos Sigma_c driver (test infrastructure only).

Restates ``SIGMA/calculate_sigma_lanczos_lowcomsym.F90z:516-779`` for one
symmetry representation (C1, ``ntrans = 1``, the case every synthetic
workload uses): start vectors ``|P_mn>``, the energy grid, the Lanczos
spectra of every band chain and the Sigma_c accumulation, plus the QP
Newton solve of ``SIGMA/printsigma.F90:97-125``.
Energies in Rydberg unless stated; ``RYD`` converts to eV.
"""
import numpy as np

from . import lanczos as L
from . import qp as Q
from .pairs import lowcomsym_pairs

RYD = 13.60569193   # shared/myconstants.F90:41


def build_cmtrx(psi_intp, cvpair):
    """``Cmtrx(mu, icv) = Psi(mu, c) * Psi(mu, v)`` (``apply_matvec_lowcomsym.F90:209-210``,
    ``calculate_sigma_lanczos.F90z:203-205``).  cvpair: (ncv, 2) 1-based (v, c)."""
    v = cvpair[:, 0] - 1
    c = cvpair[:, 1] - 1
    return psi_intp[:, c] * psi_intp[:, v]


def sqrt_r(e1, cvpair):
    """``sqrtR(icv) = (e1(c) - e1(v))**0.5`` (``calculate_sigma_lanczos_lowcomsym.F90z:547``)."""
    return (e1[cvpair[:, 1] - 1] - e1[cvpair[:, 0] - 1]) ** 0.5


def start_vectors(psi_intp, mmtrx, cmtrx, sqrtR, m1, bands, tamm_d=False):
    """``|P_mn>`` for QP band m1 and the listed bands n (1-based).

    ``calculate_sigma_lanczos_lowcomsym.F90z:578-709``:
    tmp_Cvec = psi_m * psi_n; tmp_CvecM = M tmp_Cvec; P = C^T tmp_CvecM;
    non-TDA: P *= sqrtR; pnorm2 = |P|^2.
    Returns (P (ncv, nb), pnorm2 (nb,))."""
    cmn = psi_intp[:, [m1 - 1]] * psi_intp[:, np.asarray(bands) - 1]
    cm = mmtrx @ cmn
    p = cmtrx.T @ cm
    if not tamm_d:
        p = p * sqrtR[:, None]
    pnorm2 = np.einsum("ij,ij->j", p, p)
    return p, pnorm2


def energy_grid(e1_m, deltae, nen):
    """``zz(ien) = deltae/(nen-1)*(ien-1) + e1(m) - deltae/2`` (``:520,527-530``)."""
    de = deltae / (nen - 1)
    en0 = e1_m - deltae * 0.5
    return de * np.arange(nen) + en0


def sigma_c_state(psi_intp, mmtrx, e1, nval, m1, nen, deltae, ecuts, niter,
                  polynomial, tamm_d=False, bands=None, return_ab=False, perturb=0.0,
                  lengths=None, early_exit_eps=None, reorth=False):
    """Sigma_c(omega) (Ry, complex, length nen) of QP band ``m1`` (1-based),
    summed over ``bands`` (default: all bands 1..nmem).  ``lengths``: optional
    per-band-chain Lanczos lengths; ``early_exit_eps``: per-chain exit.

    ``:713-745``: ezz = (E_n - zz)*eta_n + i*ecuts, ezz(nen+1) = 0;
    non-TDA: Sigma += (S(0) - S(ezz)) * eta_n * 2 * pnorm2 / ezz;
    TDA:     Sigma += -S(ezz) * eta_n * sqrt(2) * pnorm2.
    """
    nmem = psi_intp.shape[1]
    cvpair = lowcomsym_pairs(nval, nmem)
    cm = build_cmtrx(psi_intp, cvpair)
    sr = sqrt_r(e1, cvpair)
    if bands is None:
        bands = np.arange(1, nmem + 1)
    bands = np.asarray(bands)
    zz = energy_grid(e1[m1 - 1], deltae, nen)
    p, pnorm2 = start_vectors(psi_intp, mmtrx, cm, sr, m1, bands, tamm_d)
    pnorm = np.sqrt(pnorm2)
    eta = np.where(bands <= nval, 1.0, -1.0)
    ezz = np.zeros((nen + 1, len(bands)), dtype=np.complex128)
    ezz[:nen, :] = (-zz[:, None] + e1[bands - 1][None, :]) * eta[None, :] + 1j * ecuts
    spectra, a, b = L.lanczos_spectra_isdf(p, pnorm, ezz, niter, polynomial, cm, mmtrx, sr,
                                           tamm_d=tamm_d, perturb=perturb, lengths=lengths,
                                           early_exit_eps=early_exit_eps, reorth=reorth)
    if tamm_d:
        # 2.0**0.5 is a default-real (single precision) expression in the Fortran
        sqrt2 = float(np.sqrt(np.float32(2.0)))
        tmp = -spectra[:nen, :] * eta[None, :] * sqrt2 * pnorm2[None, :]
    else:
        tmp = ((spectra[nen:nen + 1, :] - spectra[:nen, :]) * eta[None, :] * 2.0
               * pnorm2[None, :] / ezz[:nen, :])
    sig = tmp.sum(axis=1)
    if return_ab:
        return sig, a, b, p, pnorm2
    return sig


def qp_energies(sigma_c_ry, e1, e0, qp_bands, deltae, sigx_ry, vxc_ry, xacc_ev=0.01):
    """QP energies (eV) from Sigma_c tables (Ry) -- ``printsigma.F90:97-125``."""
    out = []
    for i, m in enumerate(qp_bands):
        eqp, z, ierr = Q.qp_solve(np.asarray(sigma_c_ry[i]) * RYD, e0[m - 1] * RYD,
                                  e1[m - 1] * RYD, deltae * RYD, sigx_ry[i] * RYD,
                                  vxc_ry[i] * RYD, xacc=xacc_ev)
        out.append((eqp, z, ierr))
    return out
