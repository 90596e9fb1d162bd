"""ctypes binding of libngw_b200.so (the C ABI declared in include/ngw_b200.h).

The library is loaded from the package directory; if it is missing the import
fails loudly -- there is no CPU fallback for any entry point.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libngw_b200.so")

NGW_OK = 0
NGW_ERR_ARG = 1
NGW_ERR_OOM = 2
NGW_ERR_CUDA = 3
NGW_ERR_TIMEOUT = 4
NGW_ERR_NONFINITE = 5
NGW_ERR_BUDGET = 6
NGW_ERR_STATE = 7
NGW_ERR_NOCONV = 8

NGW_PREC_FP64 = 0
NGW_PREC_MIXED = 1

# every exported symbol of include/ngw_b200.h with (restype, argtypes)
_P = ctypes.c_void_p
_I = ctypes.c_int
_D = ctypes.c_double
SIGNATURES = {
    "ngw_version": (_I, []),
    "ngw_last_error": (ctypes.c_char_p, []),
    "ngw_session_create": (_I, [_I, ctypes.POINTER(_P)]),
    "ngw_session_destroy": (None, [_P]),
    "ngw_session_stream": (_P, [_P]),
    "ngw_set_precision": (_I, [_P, _I]),
    "ngw_session_bytes": (ctypes.c_longlong, [_P]),
    "ngw_set_isdf": (_I, [_P, _I, _I, _P, _P, _P]),
    "ngw_set_pairs": (_I, [_P, _I, _P, _P]),
    "ngw_matvec_isdf": (_I, [_P, _P, _P, _I, _I, _I]),
    "ngw_polynomial_matvec_isdf": (_I, [_P, _P, _I, _P, _P, _I, _I]),
    "ngw_lanczos_spectra_isdf": (_I, [_P, _P, _P, _I, _P, _I, _I, _P, _I, _I, _I, _P, _P, _P]),
    "ngw_lanczos_spectra_isdf_masked": (_I, [_P, _P, _P, _I, _P, _I, _I, _P, _I, _I, _I, _P, _D, _P, _P,
                                             _P]),
    "ngw_k_integrate_isdf": (_I, [_P, _I, _P, _I, _P, _I, _P]),
    "ngw_sigma_lanczos": (_I, [_P, _P, _P, _P, _P, _P]),
    "ngw_sigma_lanczos_batch": (_I, [_P, _I, _P, _P, _P]),
    "ngw_qp_newton": (_I, [_P, _I, _I, _P, _P, _P, _D, _P, _P, _D, _P, _P, _P]),
    "ngw_qp_newton_noalloc": (_I, [_I, _I, _P, _P, _P, _D, _P, _P, _D, _P, _P, _P, _P]),
    "ngw_profile_mixed_gemms": (_I, [_P, _I, _I, _P, _P]),
    "ngw_dgemm": (_I, [_I, _I, _I, _I, _I, _D, _P, _I, _P, _I, _D, _P, _I, _P, ctypes.c_longlong, _P]),
    "ngw_mixed_gemm_shapes": (_I, [_P, _I, _P]),
    "ngw_profile_dense_gemm": (_I, [_P, _I, _I, _P, _P]),
    "ngw_operator_eigenpairs": (_I, [_P, _I, _I, _I, _P, _P, _P]),
    "ngw_shell_sort": (_I, [_I, _P, _P]),
    "ngw_cvt": (_I, [_I, _P, _P, _I, _P, _I, _P, _P]),
    "ngw_cvt_device": (_I, [_P, _I, _P, _P, _I, _P, _I, _P, _P]),
    "ngw_dedup_points": (_I, [_I, _P, _P, _P, _P]),
    "ngw_build_coulomb_kernel": (_I, [_P, _I, _I, _P, _P, _I, _D, _D, _P]),
    "ngw_build_fxc_kernel": (_I, [_P, _I, _I, _P, _P, _D, _P, _P]),
    "ngw_build_isdf_kernel": (_I, [_P, _I, _I, _P, _P, _I, _P, _I, _I, _D, _D, _P, _P, _P, _P]),
    "ngw_fock_exchange": (_I, [_P, _I, _I, _P, _P, _I, _D, _D, _P, _I, _P, _I, _P]),
    "ngw_parsec_read_header": (_I, [ctypes.c_char_p, _P]),
    "ngw_parsec_read": (_I, [ctypes.c_char_p, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P]),
    "ngw_parsec_write": (_I, [ctypes.c_char_p, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P]),
    "ngw_vxc_matrix": (_I, [_P, _I, _I, _P, _P, _I, _P, _I, _P, _P]),
}


class SigmaParams(ctypes.Structure):
    """Mirror of ``ngw_sigma_params``."""
    _fields_ = [
        ("nen", _I), ("deltae", _D), ("ecuts", _D), ("niter", _I), ("npoly", _I),
        ("polynomial", _P), ("tamm_d", _I), ("nval", _I), ("nqp", _I), ("qp_bands", _P),
        ("nbands_sum", _I), ("block_chains", _I), ("cheb_lo", _D), ("cheb_hi", _D),
        ("chain_niter", _P), ("early_exit_eps", _D), ("reorth", _I),
    ]


class ParsecHeader(ctypes.Structure):
    """Mirror of ``ngw_parsec_header``."""
    _fields_ = [
        ("datelabel", ctypes.c_char * 27), ("nspin", _I), ("lcplx", _I), ("per", _I), ("ndim", _I),
        ("nwedge", _I), ("ntrans", _I), ("nstate", _I), ("nwfn", _I), ("step", _D),
        ("shift", _D * 3),
    ]


class NGWError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"ngw error {code}: {msg}")
        self.code = code


_lib = None


def lib():
    """Load the library (once).  Raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m nanogw_b200.build` "
                "(there is no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(rc):
    if rc != NGW_OK:
        msg = lib().ngw_last_error()
        raise NGWError(rc, msg.decode() if msg else "")
    return rc
