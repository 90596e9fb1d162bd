"""Oracle: CVT point selection + de-duplication (test infrastructure only).

``cvt`` wraps the C restatement of ``shared/cvt.F90:8-195`` (oracle/cvt.c);
``dedup_points`` restates ``SIGMA/sigma.F90:377-461``.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def _lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "_build", "libngw_oracle.so")
        if not os.path.exists(path):
            subprocess.check_call(["make", "-s", "-C", _HERE])
        lib = ctypes.CDLL(path)
        lib.ngw_oracle_shell_sort.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
        lib.ngw_oracle_cvt.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                       ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
        lib.ngw_oracle_cvt.restype = ctypes.c_int
        _LIB = lib
    return _LIB


def shell_sort(arr):
    """1-based ascending permutation (``shared/quicksort.f90``)."""
    a = np.ascontiguousarray(arr, dtype=np.float64)
    idx = np.zeros(len(a), dtype=np.int32)
    _lib().ngw_oracle_shell_sort(len(a), a.ctypes.data, idx.ctypes.data)
    return idx


def cvt(grid, rho, init_pts, max_iter=100000):
    """Returns (intp 1-based int32 (n_intp,), final points, iterations)."""
    g = np.ascontiguousarray(grid, dtype=np.float64)
    r = np.ascontiguousarray(rho, dtype=np.float64)
    p = np.ascontiguousarray(init_pts, dtype=np.float64).copy()
    n = p.shape[0]
    intp = np.zeros(n, dtype=np.int32)
    it = _lib().ngw_oracle_cvt(g.shape[0], g.ctypes.data, r.ctypes.data, n, p.ctypes.data,
                               int(max_iter), intp.ctypes.data)
    return intp, p, it


def dedup_points(intp, rho, ntrans=1, npes=1, trim_to_npes=False):
    """``SIGMA/sigma.F90:377-461``: keep points with mod(intp, ntrans)==0, sort
    by rho (Shell sort), drop a point when |rho - rho_next| < 1e-14 (single
    literal) in sorted order (the last of a run survives), then keep them in
    original order, trimmed to a multiple of npes for lessmemory 2-4."""
    intp = np.asarray(intp)
    tmp = intp[np.mod(intp, ntrans) == 0]
    n = len(tmp)
    if n == 0:
        return tmp.astype(np.int32)
    rho_at = np.asarray(rho)[(tmp - 1) // ntrans]
    sidx = shell_sort(rho_at) - 1
    keep = np.ones(n, dtype=bool)
    tol = float(np.float32(1.0e-14))
    ndummy = 0
    for i in range(n - 1):
        if abs(rho_at[sidx[i]] - rho_at[sidx[i + 1]]) < tol:
            keep[sidx[i]] = False
        else:
            keep[sidx[i]] = True
            ndummy += 1
    keep[sidx[n - 1]] = True
    ndummy += 1
    if trim_to_npes:
        ndummy -= ndummy % npes
    out = []
    for i in range(n):
        if keep[i]:
            out.append(tmp[i])
        if len(out) == ndummy:
            break
    return np.array(out, dtype=np.int32)
