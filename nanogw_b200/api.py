"""Python mirror of the reference's operator interface for the Lanczos GW path.

Names and argument meaning follow NanoGW:
  matvec_isdf            shared/apply_matvec.f90:25 (and _BLOCK / _lowcomsym)
  polynomial_matvec_isdf shared/apply_matvec.f90:142
  lanczos_spectra_isdf   shared/lanczos_spectra.f90:7 (and _BLOCK / _lowcomsym)
  k_integrate_isdf       shared/k_integrate_isdf.F90z:12
  calculate_sigma_lanczos SIGMA/calculate_sigma_lanczos_lowcomsym.F90z:9
  qp_newton              SIGMA/printsigma.F90:97-125
Every call goes through the C ABI of libngw_b200.so; arrays are numpy
column blocks ``(ncv, blksz)`` as in the Fortran, bands 1-based, energies in Ry.
Errors raise NGWError carrying the library's status code (the reference
calls die()).
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import NGW_PREC_FP64, NGW_PREC_MIXED, NGWError, SigmaParams, check, lib

RYD = 13.60569193   # shared/myconstants.F90:41


def _f64(a):
    return np.asfortranarray(a, dtype=np.float64)


def _p(a):
    return None if a is None else a.ctypes.data


def lowcomsym_pairs(nval, nmem):
    """(v, c) pairs in the GPU driver's order for C1 symmetry: v outer, c inner
    (``SIGMA/calculate_sigma_lanczos_lowcomsym.F90z:537-550``).  (ncv, 2) int32, 1-based."""
    v = np.repeat(np.arange(1, nval + 1), nmem - nval)
    c = np.tile(np.arange(nval + 1, nmem + 1), nval)
    return np.stack([v, c], axis=1).astype(np.int32)


def sqrt_r(e1, cvpair):
    """sqrtR(icv) = (e1(c) - e1(v))**0.5 (``calculate_sigma_lanczos_lowcomsym.F90z:547``)."""
    return (e1[cvpair[:, 1] - 1] - e1[cvpair[:, 0] - 1]) ** 0.5


class Session:
    """One device-resident ISDF operator (``type ISDF`` + pair list) on one GPU."""

    def __init__(self, device=0, precision="fp64"):
        h = ctypes.c_void_p()
        check(lib().ngw_session_create(int(device), ctypes.byref(h)))
        self._h = h
        self.device = device
        self.n_isdf = self.nmem = self.ncv = 0
        self.set_precision(precision)

    # -- lifecycle --
    def close(self):
        if getattr(self, "_h", None):
            lib().ngw_session_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def stream_ptr(self):
        return lib().ngw_session_stream(self._h)

    @property
    def device_bytes(self):
        return int(lib().ngw_session_bytes(self._h))

    def set_precision(self, precision):
        mode = {"fp64": NGW_PREC_FP64, "mixed": NGW_PREC_MIXED}[precision]
        check(lib().ngw_set_precision(self._h, mode))
        self.precision = precision

    # -- operator --
    def set_isdf(self, psi_intp, mmtrx, mxc=None):
        psi = _f64(psi_intp)
        m = _f64(mmtrx)
        x = None if mxc is None else _f64(mxc)
        self.n_isdf, self.nmem = psi.shape
        check(lib().ngw_set_isdf(self._h, self.n_isdf, self.nmem, _p(psi), _p(m), _p(x)))

    def set_pairs(self, cvpair, sqrtR):
        cv = np.ascontiguousarray(cvpair, dtype=np.int32)   # (ncv, 2) row-major == (2, ncv) Fortran
        sr = np.ascontiguousarray(sqrtR, dtype=np.float64)
        self.ncv = cv.shape[0]
        check(lib().ngw_set_pairs(self._h, self.ncv, _p(cv), _p(sr)))

    # -- reference operators --
    def matvec_isdf(self, vec, tamm_d=False):
        v = _f64(vec if np.ndim(vec) == 2 else np.asarray(vec)[:, None])
        out = np.zeros_like(v, order="F")
        check(lib().ngw_matvec_isdf(self._h, _p(v), _p(out), v.shape[0], v.shape[1], int(tamm_d)))
        return out if np.ndim(vec) == 2 else out[:, 0]

    def polynomial_matvec_isdf(self, vec, polynomial):
        v = _f64(vec if np.ndim(vec) == 2 else np.asarray(vec)[:, None])
        poly = np.ascontiguousarray(polynomial, dtype=np.float64)
        out = np.zeros_like(v, order="F")
        check(lib().ngw_polynomial_matvec_isdf(self._h, _p(poly), len(poly) - 1, _p(v), _p(out),
                                               v.shape[0], v.shape[1]))
        return out if np.ndim(vec) == 2 else out[:, 0]

    def lanczos_spectra_isdf(self, v0, v0_norm, zz, niter, polynomial=None, tamm_d=False,
                             chain_niter=None, early_exit_eps=0.0):
        """<v|1/(zz - p(H))|v> per column.  chain_niter: optional per-chain
        Lanczos lengths; early_exit_eps > 0: a chain stops when |b_k| < eps
        (the single-vector reference form uses 1e-8)."""
        v = _f64(v0 if np.ndim(v0) == 2 else np.asarray(v0)[:, None])
        nb = v.shape[1]
        nrm = np.ascontiguousarray(np.broadcast_to(np.asarray(v0_norm, dtype=np.float64), (nb,)))
        z = np.asfortranarray(np.asarray(zz, dtype=np.complex128).reshape(-1, nb) if np.ndim(zz) == 2
                              else np.repeat(np.asarray(zz, dtype=np.complex128)[:, None], nb, 1))
        nz = z.shape[0]
        spec = np.zeros((nz, nb), dtype=np.complex128, order="F")
        a = np.zeros((niter, nb), order="F")
        b = np.zeros((niter, nb), order="F")
        if polynomial is None:
            poly = np.zeros(2)
            npoly = 1
        else:
            poly = np.ascontiguousarray(polynomial, dtype=np.float64)
            npoly = len(poly) - 1
        ln = None if chain_niter is None else np.ascontiguousarray(chain_niter, dtype=np.int32)
        if ln is None and not early_exit_eps:
            check(lib().ngw_lanczos_spectra_isdf(self._h, _p(v), _p(nrm), v.shape[0], _p(z), nz,
                                                 int(niter), _p(poly), npoly, nb, int(tamm_d), _p(spec),
                                                 _p(a), _p(b)))
        else:
            check(lib().ngw_lanczos_spectra_isdf_masked(self._h, _p(v), _p(nrm), v.shape[0], _p(z), nz,
                                                        int(niter), _p(poly), npoly, nb, int(tamm_d),
                                                        _p(ln), float(early_exit_eps), _p(spec), _p(a),
                                                        _p(b)))
        return spec, a, b

    def k_integrate_isdf(self, kflag, rows, cols):
        r = np.ascontiguousarray(rows, dtype=np.int32)
        c = np.ascontiguousarray(cols, dtype=np.int32)
        out = np.zeros((len(r), len(c)), order="F")
        check(lib().ngw_k_integrate_isdf(self._h, int(kflag), _p(r), len(r), _p(c), len(c), _p(out)))
        return out

    def _sigma_params(self, e1, nval, qp_bands, nen, deltae, ecuts, niter, polynomial, tamm_d=False,
                      nbands_sum=0, block_chains=0, cheb=(0.0, 0.0), chain_niter=None,
                      early_exit_eps=0.0, reorth=False):
        """ngw_sigma_params for one request, with the arrays it points to."""
        e = np.ascontiguousarray(e1, dtype=np.float64)
        qp = np.ascontiguousarray(qp_bands, dtype=np.int32)
        poly = np.ascontiguousarray(polynomial if polynomial is not None else [1.0, 0.0],
                                    dtype=np.float64)
        nbs = nbands_sum if nbands_sum > 0 else self.nmem
        prm = SigmaParams(nen=int(nen), deltae=float(deltae), ecuts=float(ecuts), niter=int(niter),
                          npoly=len(poly) - 1, polynomial=_p(poly), tamm_d=int(tamm_d),
                          nval=int(nval), nqp=len(qp), qp_bands=_p(qp), nbands_sum=int(nbands_sum),
                          block_chains=int(block_chains), cheb_lo=float(cheb[0]),
                          cheb_hi=float(cheb[1]), chain_niter=None,
                          early_exit_eps=float(early_exit_eps), reorth=int(bool(reorth)))
        ln = None
        if chain_niter is not None:
            ln = np.ascontiguousarray(chain_niter, dtype=np.int32).reshape(-1)
            if ln.size != len(qp) * nbs:
                raise ValueError("chain_niter must have nqp * nbands_sum entries")
            prm.chain_niter = _p(ln)
        sig = np.zeros((nen, len(qp)), dtype=np.complex128, order="F")
        return prm, e, sig, (qp, poly, ln), nbs

    def calculate_sigma_lanczos(self, e1, nval, qp_bands, nen, deltae, ecuts, niter, polynomial,
                                tamm_d=False, nbands_sum=0, block_chains=0, cheb=(0.0, 0.0),
                                return_ab=False, chain_niter=None, early_exit_eps=0.0, reorth=False):
        """Sigma_c(omega) (Ry) for each QP band: complex array (nen, nqp).
        chain_niter: optional (nqp, nbands_sum) per-chain Lanczos lengths
        (1..niter); early_exit_eps > 0 stops a chain when |b_k| < eps;
        reorth: full reorthogonalisation of every chain (not in the reference)."""
        prm, e, sig, keep, nbs = self._sigma_params(e1, nval, qp_bands, nen, deltae, ecuts, niter,
                                                    polynomial, tamm_d, nbands_sum, block_chains,
                                                    cheb, chain_niter, early_exit_eps, reorth)
        a = b = None
        if return_ab:
            a = np.zeros((niter, nbs * sig.shape[1]), order="F")
            b = np.zeros((niter, nbs * sig.shape[1]), order="F")
        check(lib().ngw_sigma_lanczos(self._h, ctypes.byref(prm), _p(e), _p(sig), _p(a), _p(b)))
        if return_ab:
            return sig, a, b
        return sig

    def qp_newton(self, sigma_c_ev, e1_ev, e0_ev, deltae_ev, sigx_ev, vxc_ev, xacc_ev=0.01):
        s = np.asfortranarray(sigma_c_ev, dtype=np.complex128)
        nen, nqp = s.shape
        f = lambda x: np.ascontiguousarray(np.broadcast_to(np.asarray(x, dtype=np.float64), (nqp,)))
        e1, e0, sx, vx = f(e1_ev), f(e0_ev), f(sigx_ev), f(vxc_ev)
        eqp = np.zeros(nqp)
        z = np.zeros(nqp)
        ierr = np.zeros(nqp, dtype=np.int32)
        check(lib().ngw_qp_newton(self._h, nqp, nen, _p(s), _p(e1), _p(e0), float(deltae_ev), _p(sx),
                                  _p(vx), float(xacc_ev), _p(eqp), _p(z), _p(ierr)))
        return eqp, z, ierr

    def profile_mixed_gemms(self, nb, reps=20):
        """(us_gemm1, us_gemm2): mean device time of one launch of each GEMM."""
        t1 = np.zeros(1)
        t2 = np.zeros(1)
        check(lib().ngw_profile_mixed_gemms(self._h, int(nb), int(reps), _p(t1), _p(t2)))
        return float(t1[0]), float(t2[0])

    def profile_dense_gemm(self, nb, reps=20):
        """(us, [M, N, K, N tile, variant]) of the dense p(C) GEMM, or None when
        the session's last mixed plan used the factored form."""
        us = np.zeros(1)
        sh = np.zeros(5, dtype=np.int32)
        rc = lib().ngw_profile_dense_gemm(self._h, int(nb), int(reps), _p(us), _p(sh))
        if rc == _lib.NGW_ERR_STATE:
            return None
        check(rc)
        return float(us[0]), [int(x) for x in sh]

    def mixed_gemm_shapes(self, nb):
        sh = np.zeros(13, dtype=np.int32)
        check(lib().ngw_mixed_gemm_shapes(self._h, int(nb), _p(sh)))
        return [int(x) for x in sh]

    def operator_eigenpairs(self, kmax=16, msteps=240, tamm_d=False):
        """Largest Ritz values of the Casida operator (C, or A with TDA) and
        their residual bounds from an FP64 Lanczos run of msteps steps with
        full reorthogonalisation (the pairs the mixed path deflates)."""
        vals = np.zeros(kmax)
        res = np.zeros(kmax)
        cnt = ctypes.c_int(0)
        check(lib().ngw_operator_eigenpairs(self._h, int(bool(tamm_d)), int(msteps), int(kmax), _p(vals),
                                            _p(res), ctypes.byref(cnt)))
        return vals[: cnt.value].copy(), res[: cnt.value].copy()

    def build_fxc_kernel(self, zeta, rho, h, return_fxc=False):
        """M_xc = zeta^T (f_xc * zeta) / hcub with the LDA f_xc of rho (Ry)."""
        zt = _f64(zeta)
        r = np.ascontiguousarray(rho, dtype=np.float64)
        ngrid, n_isdf = zt.shape
        m = np.zeros((n_isdf, n_isdf), order="F")
        f = np.zeros(ngrid) if return_fxc else None
        check(lib().ngw_build_fxc_kernel(self._h, ngrid, n_isdf, _p(zt), _p(r), float(h), _p(m), _p(f)))
        return (m, f) if return_fxc else m

    def build_isdf_kernel(self, psi, grid_idx, intp, mv, nfft, h, trunc, rho=None):
        """ISDF fit + kernel blocks on the device.  Returns (psi_intp, M_C, M_xc or None)."""
        ps = _f64(psi)
        g = np.ascontiguousarray(grid_idx, dtype=np.int32)
        ip = np.ascontiguousarray(intp, dtype=np.int32)
        ngrid, nmem = ps.shape
        n_isdf = len(ip)
        pi = np.zeros((n_isdf, nmem), order="F")
        m = np.zeros((n_isdf, n_isdf), order="F")
        r = None if rho is None else np.ascontiguousarray(rho, dtype=np.float64)
        mx = None if rho is None else np.zeros((n_isdf, n_isdf), order="F")
        check(lib().ngw_build_isdf_kernel(self._h, ngrid, nmem, _p(ps), _p(g), n_isdf, _p(ip), int(mv),
                                          int(nfft), float(h), float(trunc), _p(r), _p(pi), _p(m),
                                          _p(mx)))
        return pi, m, mx

    def fock_exchange(self, psi, grid_idx, nfft, h, trunc, occ, sig_bands, ntrans=1):
        """Bare exchange matrix Sigma_x (Ry) between ``sig_bands`` (1-based)."""
        ps = _f64(psi)
        g = np.ascontiguousarray(grid_idx, dtype=np.int32)
        oc = np.ascontiguousarray(occ, dtype=np.float64)
        sb = np.ascontiguousarray(sig_bands, dtype=np.int32)
        kx = np.zeros((len(sb), len(sb)), order="F")
        check(lib().ngw_fock_exchange(self._h, ps.shape[0], ps.shape[1], _p(ps), _p(g), int(nfft),
                                      float(h), float(trunc), _p(oc), len(sb), _p(sb), int(ntrans),
                                      _p(kx)))
        return kx

    def vxc_matrix(self, psi, rho, sig_bands, ntrans=1):
        """(V_xc, V_x) matrices (Ry) of the LDA between ``sig_bands``."""
        ps = _f64(psi)
        r = np.ascontiguousarray(rho, dtype=np.float64)
        sb = np.ascontiguousarray(sig_bands, dtype=np.int32)
        v = np.zeros((len(sb), len(sb)), order="F")
        vx = np.zeros((len(sb), len(sb)), order="F")
        check(lib().ngw_vxc_matrix(self._h, ps.shape[0], ps.shape[1], _p(ps), _p(r), len(sb), _p(sb),
                                   int(ntrans), _p(v), _p(vx)))
        return v, vx

    def build_coulomb_kernel(self, zeta, grid_idx, nfft, h, trunc):
        zt = _f64(zeta)
        g = np.ascontiguousarray(grid_idx, dtype=np.int32)
        ngrid, n_isdf = zt.shape
        m = np.zeros((n_isdf, n_isdf), order="F")
        check(lib().ngw_build_coulomb_kernel(self._h, ngrid, n_isdf, _p(zt), _p(g), int(nfft), float(h),
                                             float(trunc), _p(m)))
        return m


def sigma_lanczos_batch(sessions, requests):
    """Sigma_c of several molecules in one graph launch (``ngw_sigma_lanczos_batch``).
    sessions: Session objects (one molecule each, same device); requests: one
    dict of ``calculate_sigma_lanczos`` arguments per session (no return_ab).
    Returns the list of Sigma_c arrays, each bit-identical to the single call."""
    if len(sessions) != len(requests) or not sessions:
        raise ValueError("one request per session")
    built = [s._sigma_params(**r) for s, r in zip(sessions, requests)]
    n = len(sessions)
    params = (SigmaParams * n)(*[b[0] for b in built])
    hs = (ctypes.c_void_p * n)(*[s._h for s in sessions])
    e1s = (ctypes.c_void_p * n)(*[_p(b[1]) for b in built])
    sigs = (ctypes.c_void_p * n)(*[_p(b[2]) for b in built])
    check(lib().ngw_sigma_lanczos_batch(hs, n, params, e1s, sigs))
    return [b[2] for b in built]
