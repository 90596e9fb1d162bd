"""nanogw_b200 -- B200-native (sm_100a) ISDF-Lanczos GW self-energy path.

Drop-in for NanoGW's Lanczos Sigma_c path (matvec_isdf, lanczos_spectra_isdf,
k_integrate_isdf, calculate_sigma_lanczos) through the C ABI in
``include/ngw_b200.h``; the Python classes here are a thin mirror of it.
"""
from ._lib import NGWError, NGW_PREC_FP64, NGW_PREC_MIXED  # noqa: F401
from .api import RYD, Session, lowcomsym_pairs, sigma_lanczos_batch, sqrt_r  # noqa: F401

__all__ = ["Session", "NGWError", "RYD", "lowcomsym_pairs", "sigma_lanczos_batch", "sqrt_r"]
